// vrt_oracle.cpp -- CPU oracle (TEST INFRASTRUCTURE ONLY; see oracle.h).
//
// Sequential restatement of the reference's volumetric GLSL, templated on the
// arithmetic type T (float to follow the GPU's float paths draw for draw,
// double for the fine references).  Every function cites the reference file
// and lines it restates.  Parity with the reference itself is UNPINNED: the
// reference has no golden vectors and its shaders need Vulkan, which is absent.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <omp.h>

namespace {

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).  Replaces the reference's Tausworthe+LCG state
// (include/randoms.h:6-59); the float conversion below keeps the reference's
// 23-mantissa-bit trick (include/randoms.h:51-56).
// ---------------------------------------------------------------------------
inline void philox(uint32_t k0, uint32_t k1, const uint32_t c[4], uint32_t o[4]) {
    uint32_t x0 = c[0], x1 = c[1], x2 = c[2], x3 = c[3];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * x0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * x2;
        uint32_t y0 = (uint32_t)(p1 >> 32) ^ x1 ^ k0;
        uint32_t y1 = (uint32_t)p1;
        uint32_t y2 = (uint32_t)(p0 >> 32) ^ x3 ^ k1;
        uint32_t y3 = (uint32_t)p0;
        x0 = y0; x1 = y1; x2 = y2; x3 = y3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    o[0] = x0; o[1] = x1; o[2] = x2; o[3] = x3;
}

// Draw k of stream s of path p = word (k & 3) of philox(seed, {k>>2, p_lo, s, p_hi}).
// Every transmittance estimate draws from a stream of its own, forked from the
// stream that requests it: the j-th fork of stream s is stream s + 2(j+1)
// (stream 0 is the path, stream 1 the branch stream of the DRT adjoint, so the
// two families never meet).  Draws stay i.i.d. uniforms, as in the reference's
// single Tausworthe stream, and re-forking from a saved state replays a shadow
// ray exactly (the reference's SAVE_SEED(before_transmittance)).
struct Rng {
    uint32_t k0, k1, plo, phi, stream, n, ntr;
    Rng(uint64_t seed, uint64_t path, uint32_t s)
        : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), plo((uint32_t)path),
          phi((uint32_t)(path >> 32)), stream(s), n(0), ntr(0) {}
    Rng fork() {
        Rng r = *this;
        r.stream = stream + 2u * (1u + ntr);
        r.n = 0;
        r.ntr = 0;
        ++ntr;
        return r;
    }
    uint32_t u32() {
        uint32_t c[4] = {n >> 2, plo, stream, phi}, o[4];
        philox(k0, k1, c, o);
        uint32_t v = o[n & 3];
        ++n;
        return v;
    }
    float uniform() {  // randoms.h:51-56: uintBitsToFloat(v & 0x7FFFFF | 0x3F800000) - 1
        uint32_t b = (u32() & 0x007FFFFFu) | 0x3F800000u;
        float f;
        std::memcpy(&f, &b, 4);
        return f - 1.0f;
    }
    void advance() { ++n; }  // randoms.h:35-41 advance_random
    // stream s of the same path and key (the collision integrators give the
    // collision sampler, its adjoint and every exitance evaluation a stream)
    Rng with_stream(uint32_t s) const {
        Rng r = *this;
        r.stream = s;
        r.n = 0;
        r.ntr = 0;
        return r;
    }
    // The DRTQ adjoint's scatter term of segment k (0: the primary ray's, k:
    // the one after the k-th scattering vertex) draws from a stream of its
    // own: stream s + 1 of the path id with k + 1 in bits 40-63 (path ids
    // below 2^40, k + 1 below 2^24).  No term depends on another's draws, so
    // the terms can run in any order.
    Rng segment_stream(uint32_t k) const {
        Rng r = *this;
        r.phi = phi | ((k + 1u) << 8);
        r.stream = stream + 1u;
        r.n = 0;
        r.ntr = 0;
        return r;
    }
};

template <typename T> struct V3 {
    T x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    explicit V3(T a) : x(a), y(a), z(a) {}
    static V3 load(const float* p) { return V3((T)p[0], (T)p[1], (T)p[2]); }
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <typename T> V3<T> operator+(V3<T> a, V3<T> b) { return V3<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T> V3<T> operator-(V3<T> a, V3<T> b) { return V3<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T> V3<T> operator*(V3<T> a, V3<T> b) { return V3<T>(a.x * b.x, a.y * b.y, a.z * b.z); }
template <typename T> V3<T> operator/(V3<T> a, V3<T> b) { return V3<T>(a.x / b.x, a.y / b.y, a.z / b.z); }
template <typename T> V3<T> operator*(V3<T> a, T s) { return V3<T>(a.x * s, a.y * s, a.z * s); }
template <typename T> V3<T> operator*(T s, V3<T> a) { return V3<T>(s * a.x, s * a.y, s * a.z); }
template <typename T> V3<T> operator/(V3<T> a, T s) { return V3<T>(a.x / s, a.y / s, a.z / s); }
template <typename T> V3<T> operator-(V3<T> a) { return V3<T>(-a.x, -a.y, -a.z); }
template <typename T> V3<T>& operator+=(V3<T>& a, V3<T> b) { a = a + b; return a; }
template <typename T> V3<T>& operator-=(V3<T>& a, V3<T> b) { a = a - b; return a; }
template <typename T> V3<T>& operator*=(V3<T>& a, V3<T> b) { a = a * b; return a; }
template <typename T> V3<T>& operator*=(V3<T>& a, T s) { a = a * s; return a; }
template <typename T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> V3<T> cross(V3<T> a, V3<T> b) {
    return V3<T>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template <typename T> V3<T> normalize(V3<T> a) { return a / std::sqrt(dot(a, a)); }
template <typename T> bool all_less(V3<T> a, T e) { return a.x < e && a.y < e && a.z < e; }
template <typename T> T mix(T a, T b, T t) { return a * (T(1) - t) + b * t; }
template <typename T> T vmin(T a, T b) { return b < a ? b : a; }  // GLSL min
template <typename T> T vmax(T a, T b) { return a < b ? b : a; }  // GLSL max

template <typename T> struct K {
    static constexpr T pi = T(3.1415926535897932384626433832795);
    static constexpr T two_pi = T(6.283185307179586476925286766559);
};

inline void atomic_add(float* p, float v) {
#pragma omp atomic
    *p += v;
}

struct Counters {
    int64_t paths = 0, vertices = 0, steps = 0;
};

// Optical distance of the current free flight.  With a piecewise-constant
// majorant the flight continues across a majorant-brick face with the optical
// depth it has left (exponential lengths are memoryless), so a new draw is
// taken only after the previous one ended at a candidate collision or at the
// end of the segment.  With the reference's constant majorant (distance 1e6)
// no flight ever crosses a face and every step draws, as in the reference.
template <typename T> struct Scene;

// Majorant bricks along one straight segment (majorant-grid mode): a 3D DDA
// over the brick grid started at the segment's first query.  The brick of the
// start point is chosen with the 1e-4-brick nudge of Scene::majorant, the face
// distances use correctly rounded reciprocals, and outside the grid's box the
// bound is 0.  A segment that never reaches the grid (tested at its start)
// gets no face to cross; one that leaves it walks on through bound-0 bricks
// until it ends.  With the constant majorant it is inert.
template <typename T> struct BrickWalk {
    bool live = false;
    int c[3] = {0, 0, 0}, st[3] = {0, 0, 0};
    T tn[3] = {0, 0, 0}, dt[3] = {0, 0, 0}, t = 0, m = 0;
    void reset() { live = false; }
    T lookup(const orc_scene& s) const {
        for (int i = 0; i < 3; ++i)
            if (c[i] < 0 || c[i] >= s.maj_dims[i]) return T(0);
        return (T)s.maj_grid[((int64_t)c[2] * s.maj_dims[1] + c[1]) * s.maj_dims[0] + c[0]];
    }
    void init(const orc_scene& s, V3<T> x, V3<T> w) {
        live = true;
        t = T(0);
        const T inf = std::numeric_limits<T>::infinity();
        for (int i = 0; i < 3; ++i) {
            T q = (x[i] - (T)s.bmin[i]) * (T)s.maj_scale[i];
            T dq = w[i] * (T)s.maj_scale[i];
            if (dq > T(0)) {
                c[i] = (int)std::floor(q + T(1e-4)); st[i] = 1;
                T rv = T(1) / dq;
                tn[i] = (T(c[i] + 1) - q) * rv; dt[i] = rv;
            } else if (dq < T(0)) {
                c[i] = (int)std::floor(q - T(1e-4)); st[i] = -1;
                T rv = T(1) / dq;
                tn[i] = (T(c[i]) - q) * rv; dt[i] = -rv;
            } else {
                c[i] = (int)std::floor(q); st[i] = 0; tn[i] = inf; dt[i] = inf;
            }
        }
        m = lookup(s);
        if (never_enters(s)) tn[0] = tn[1] = tn[2] = inf;  // a segment that never reaches the grid: no face
    }
    int axis() const { return (tn[0] <= tn[1] && tn[0] <= tn[2]) ? 0 : (tn[1] <= tn[2] ? 1 : 2); }
    bool never_enters(const orc_scene& s) const {
        for (int i = 0; i < 3; ++i)
            if ((c[i] < 0 && st[i] <= 0) || (c[i] >= s.maj_dims[i] && st[i] >= 0)) return true;
        return false;
    }
    T query(const orc_scene& s, V3<T> x, V3<T> w, T& md) {
        if (s.majorant_mode == 0) { md = T(1000000.0); return (T)s.global_majorant; }
        if (!live) init(s, x, w);
        md = tn[axis()] - t;
        return m;
    }
    void advance(const orc_scene& s) {
        if (!live) return;
        int a = axis();
        t = tn[a];
        tn[a] += dt[a];
        c[a] += st[a];
        m = lookup(s);
    }
    void move(T dist) { t += dist; }
};

template <typename T> struct Flight {
    T tau = T(-1);
    int it = 0;
    BrickWalk<T> bk;  // majorant bricks of the current segment
    T sample(Rng& rng) {
        if (tau < T(0)) tau = -std::log(T(1) - (T)rng.uniform());
        return tau;
    }
    void cross(T m, T md) { tau -= m * md; }
    void used() { tau = T(-1); }
};

// ---------------------------------------------------------------------------
// include/maths.h:11-26 intersect_ray_box and :28-38 ray_box_intersection
// ---------------------------------------------------------------------------
template <typename T> V3<T> unparallel(V3<T> w) {
    const T e = T(0.000001);
    w.x = std::abs(w.x) <= e ? e : w.x;
    w.y = std::abs(w.y) <= e ? e : w.y;
    w.z = std::abs(w.z) <= e ? e : w.z;
    return w;
}
template <typename T>
void ray_box_intersection(V3<T> x, V3<T> w, V3<T> bmin, V3<T> bmax, T& tMin, T& tMax) {
    w = unparallel(w);
    V3<T> cmin = (bmin - x) / w, cmax = (bmax - x) / w;
    tMin = vmax(vmax(vmin(cmin.x, cmax.x), vmin(cmin.y, cmax.y)), vmin(cmin.z, cmax.z));
    tMax = vmin(vmin(vmax(cmin.x, cmax.x), vmax(cmin.y, cmax.y)), vmax(cmin.z, cmax.z));
}
template <typename T>
bool intersect_ray_box(V3<T> x, V3<T> w, V3<T> bmin, V3<T> bmax, T& tMin, T& tMax) {
    ray_box_intersection(x, w, bmin, bmax, tMin, tMax);
    tMin = vmax(T(0), tMin);
    if (tMax <= tMin || tMax <= T(0)) return false;
    return true;
}

// ---------------------------------------------------------------------------
// Scene accessors: the vr_*.h shims (include/vr_boundary.h, vr_sigma.h, ...)
// bound to the sub-maps this path lowers: RayBoxIntersection, Grid3D, const.
// ---------------------------------------------------------------------------
template <typename T> struct Scene {
    const orc_scene& s;
    explicit Scene(const orc_scene& sc) : s(sc) {}

    // include/vr_boundary.h:1-11 over RayBoxIntersection (_maps.py:4128-4154)
    bool boundary(V3<T> x, V3<T> w, T& tMin, T& tMax) const {
        ray_box_intersection(x, w, V3<T>::load(s.box_min), V3<T>::load(s.box_max), tMin, tMax);
        tMin = vmax(T(0), tMin);
        return !(tMax < tMin) && tMax == tMax && tMin == tMin;  // a NaN interval is a miss
    }

    // include/maps/grid3d.h:6-37 (Grid3D FORWARD), channel count C
    void grid_fw(const orc_grid& g, V3<T> c, T* out) const {
        V3<T> nc((c.x - (T)s.bmin[0]) * (T)s.inv_bsize[0], (c.y - (T)s.bmin[1]) * (T)s.inv_bsize[1],
                 (c.z - (T)s.bmin[2]) * (T)s.inv_bsize[2]);
        grid_fw_n(g, nc, out);
    }
    static void grid_fw_n(const orc_grid& g, V3<T> nc, T* out) {
        for (int i = 0; i < g.C; ++i) out[i] = T(0);
        if (nc.x < T(0) || nc.y < T(0) || nc.z < T(0) || nc.x >= T(1) || nc.y >= T(1) || nc.z >= T(1)) return;
        const int dx = g.W - 1, dy = g.H - 1, dz = g.D - 1;
        V3<T> gc(nc.x * T(dx), nc.y * T(dy), nc.z * T(dz));
        V3<T> a(gc.x - std::floor(gc.x), gc.y - std::floor(gc.y), gc.z - std::floor(gc.z));
        int px = std::min(std::max((int)gc.x, 0), dx - 1);
        int py = std::min(std::max((int)gc.y, 0), dy - 1);
        int pz = std::min(std::max((int)gc.z, 0), dz - 1);
        const T one(1);
        const int ox[8] = {0, 1, 0, 1, 0, 1, 0, 1}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1}, oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
        for (int k = 0; k < 8; ++k) {
            T wx = ox[k] ? a.x : one - a.x, wy = oy[k] ? a.y : one - a.y, wz = oz[k] ? a.z : one - a.z;
            T wt = wx * wy * wz;
            const float* src = g.data + ((((int64_t)(pz + oz[k]) * g.H + (py + oy[k])) * g.W + (px + ox[k])) * g.C);
            for (int i = 0; i < g.C; ++i) out[i] += (T)src[i] * wt;
        }
    }
    // include/maps/grid3d.h:39-75 (Grid3D BACKWARD)
    void grid_bw(const orc_grid& g, V3<T> c, const T* dout) const {
        if (!g.grad) return;
        V3<T> nc((c.x - (T)s.bmin[0]) * (T)s.inv_bsize[0], (c.y - (T)s.bmin[1]) * (T)s.inv_bsize[1],
                 (c.z - (T)s.bmin[2]) * (T)s.inv_bsize[2]);
        grid_bw_n(g, nc, dout);
    }
    static void grid_bw_n(const orc_grid& g, V3<T> nc, const T* dout) {
        if (!g.grad) return;
        if (nc.x < T(0) || nc.y < T(0) || nc.z < T(0) || nc.x >= T(1) || nc.y >= T(1) || nc.z >= T(1)) return;
        const int dx = g.W - 1, dy = g.H - 1, dz = g.D - 1;
        V3<T> gc(nc.x * T(dx), nc.y * T(dy), nc.z * T(dz));
        V3<T> a(gc.x - std::floor(gc.x), gc.y - std::floor(gc.y), gc.z - std::floor(gc.z));
        int px = std::min(std::max((int)gc.x, 0), dx - 1);
        int py = std::min(std::max((int)gc.y, 0), dy - 1);
        int pz = std::min(std::max((int)gc.z, 0), dz - 1);
        const T one(1);
        const int ox[8] = {0, 1, 0, 1, 0, 1, 0, 1}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1}, oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
        for (int i = 0; i < g.C; ++i)
            for (int k = 0; k < 8; ++k) {
                T wx = ox[k] ? a.x : one - a.x, wy = oy[k] ? a.y : one - a.y, wz = oz[k] ? a.z : one - a.z;
                float* dst = g.grad + ((((int64_t)(pz + oz[k]) * g.H + (py + oy[k])) * g.W + (px + ox[k])) * g.C);
                atomic_add(dst + i, (float)(dout[i] * wx * wy * wz));
            }
    }

    // include/vr_sigma.h:1-11 over Grid3D
    T sigma(V3<T> x) const { T v; grid_fw(s.sigma, x, &v); return v; }
    void sigma_bw(V3<T> x, T dL) const { grid_bw(s.sigma, x, &dL); }

    // include/vr_scattering_albedo.h over const or Grid3D (C==1 promoted to 3)
    V3<T> albedo(V3<T> x) const {
        if (!s.albedo_is_grid) return V3<T>::load(s.albedo_const);
        T v[3];
        grid_fw(s.albedo, x, v);
        return s.albedo.C == 1 ? V3<T>(v[0]) : V3<T>(v[0], v[1], v[2]);
    }
    void albedo_bw(V3<T> x, V3<T> dL) const {
        if (!s.albedo_is_grid || !s.albedo.grad) return;
        if (s.albedo.C == 1) { T g = dL.x + dL.y + dL.z; grid_bw(s.albedo, x, &g); }
        else { T g[3] = {dL.x, dL.y, dL.z}; grid_bw(s.albedo, x, g); }
    }
    V3<T> emission() const { return V3<T>::load(s.emission); }
    // include/vr_emission.h over const or a Grid3D of emission (C 1 or 3,
    // sigma's box; the collision integrators' exitance radiance)
    V3<T> emission_at(V3<T> x) const {
        if (!s.emission_is_grid) return emission();
        T v[3];
        grid_fw(s.emission_grid, x, v);
        return s.emission_grid.C == 1 ? V3<T>(v[0]) : V3<T>(v[0], v[1], v[2]);
    }
    void emission_bw(V3<T> x, V3<T> dL) const {
        if (!s.emission_is_grid || !s.emission_grid.grad) return;
        if (s.emission_grid.C == 1) { T g = dL.x + dL.y + dL.z; grid_bw(s.emission_grid, x, &g); }
        else { T g[3] = {dL.x, dL.y, dL.z}; grid_bw(s.emission_grid, x, g); }
    }
    // the environment radiance towards w: const env, or Image2D(image).after(xr_projection)
    // (_objects.py:165-172; include/maps/image2d.h:1-26 with the default box [-1, 1]^2;
    // include/maths.h:172-178 dir2xr)
    V3<T> environment(V3<T> w) const {
        if (s.env_mode == 0) return V3<T>::load(s.env);
        if (w.x == T(0) && w.z == T(0)) w.x += T(0.0000001);
        const T cx = std::atan2(w.x, w.z) * (T(1) / K<T>::pi);
        const T cy = T(-2) * std::asin(std::min(std::max(w.y, T(-1)), T(1))) * (T(1) / K<T>::pi);
        const T nx = std::min(std::max((cx - T(-1)) * T(0.5), T(0)), T(1));
        const T ny = std::min(std::max((cy - T(-1)) * T(0.5), T(0)), T(1));
        const int H = s.env_hw[0], W = s.env_hw[1];
        const T gx = nx * T(W) - T(0.5), gy = ny * T(H) - T(0.5);
        const T fx = std::floor(gx), fy = std::floor(gy);
        const int px = (int)fx, py = (int)fy;
        const T ax = gx - fx, ay = gy - fy;
        const int x0 = std::min(std::max(px, 0), W - 1), x1 = std::min(std::max(px + 1, 0), W - 1);
        const int y0 = std::min(std::max(py, 0), H - 1), y1 = std::min(std::max(py + 1, 0), H - 1);
        const float* r0 = s.env_image + 3 * ((int64_t)y0 * W);
        const float* r1 = s.env_image + 3 * ((int64_t)y1 * W);
        V3<T> o;
        for (int c = 0; c < 3; ++c)
            o[c] = mix(mix((T)r0[3 * x0 + c], (T)r0[3 * x1 + c], ax), mix((T)r1[3 * x0 + c], (T)r1[3 * x1 + c], ax), ay);
        return o;
    }

    // include/vr_majorant.h:1-7.  Mode 0: const[[max sigma, 1e6]] (_objects.py:96-101).
    // Mode 1 (extension): majorant grid of bricks; returns the brick's bound and
    // the distance to leave the brick along w.
    // Outside the grid's box the bound is 0 (Grid3D is zero there) and the
    // distance is the one to (re-)enter the box, or 1e6 when w leaves it.
    T majorant(V3<T> x, V3<T> w, T& md) const {
        if (s.majorant_mode == 0) { md = T(1000000.0); return (T)s.global_majorant; }
        const T inf = std::numeric_limits<T>::infinity();
        bool inside = true;
        for (int i = 0; i < 3; ++i) {
            T q = (x[i] - (T)s.bmin[i]) * (T)s.maj_scale[i];
            if (!(q >= T(0) && q <= T(s.maj_dims[i]))) inside = false;
        }
        if (!inside) {
            T tn = -inf, tf = inf;
            for (int i = 0; i < 3; ++i) {
                T q = (x[i] - (T)s.bmin[i]) * (T)s.maj_scale[i];
                T v = w[i] * (T)s.maj_scale[i];
                if (v != T(0)) {
                    T rv = T(1) / v;
                    T a = (T(0) - q) * rv, b = (T(s.maj_dims[i]) - q) * rv;
                    tn = vmax(tn, vmin(a, b));
                    tf = vmin(tf, vmax(a, b));
                } else if (!(q >= T(0) && q <= T(s.maj_dims[i]))) {
                    tn = inf;
                }
            }
            md = (tn < tf && tn > T(0)) ? vmax(tn, T(1e-6)) : T(1000000.0);
            return T(0);
        }
        int c[3];
        T dist = inf;
        for (int i = 0; i < 3; ++i) {
            T q = (x[i] - (T)s.bmin[i]) * (T)s.maj_scale[i];
            T nudge = w[i] > T(0) ? T(1e-4) : (w[i] < T(0) ? T(-1e-4) : T(0));
            int ci = (int)std::floor(q + nudge);
            ci = std::min(std::max(ci, 0), s.maj_dims[i] - 1);
            c[i] = ci;
            T v = w[i] * (T)s.maj_scale[i];
            T rv = T(1) / v;  // face distances use a correctly rounded reciprocal
            T di = v > T(0) ? (T(ci + 1) - q) * rv : (v < T(0) ? (T(ci) - q) * rv : std::numeric_limits<T>::infinity());
            dist = vmin(dist, di);
        }
        md = vmax(dist, T(1e-6));
        return (T)s.maj_grid[((int64_t)c[2] * s.maj_dims[1] + c[1]) * s.maj_dims[0] + c[0]];
    }

    // include/vr_sigma_grid.h:1-7 sigma_at (DDA-side lookup, clamps to [0,dim], no zeroing)
    T sigma_at(int x, int y, int z) const {
        const orc_grid& g = s.sigma;
        x = std::min(std::max(x, 0), g.W - 1);
        y = std::min(std::max(y, 0), g.H - 1);
        z = std::min(std::max(z, 0), g.D - 1);
        return (T)g.data[(((int64_t)z * g.H + y) * g.W + x) * g.C];
    }
    void sigma_at_bw(int x, int y, int z, T dL) const {
        const orc_grid& g = s.sigma;
        x = std::min(std::max(x, 0), g.W - 1);
        y = std::min(std::max(y, 0), g.H - 1);
        z = std::min(std::max(z, 0), g.D - 1);
        atomic_add(g.grad + (((int64_t)z * g.H + y) * g.W + x) * g.C, (float)dL);
    }
};

// include/vr_sigma_grid.h:18-27 interpolated_sigma, s[dz][dy][dx]
template <typename T> T interpolated_sigma(V3<T> a, const T s[2][2][2]) {
    return mix(mix(mix(s[0][0][0], s[0][0][1], a.x), mix(s[0][1][0], s[0][1][1], a.x), a.y),
               mix(mix(s[1][0][0], s[1][0][1], a.x), mix(s[1][1][0], s[1][1][1], a.x), a.y), a.z);
}
// include/vr_sigma_grid.h:29-39 interpolated_sigma_bw
template <typename T> void interpolated_sigma_bw(V3<T> a, T dL, T g[2][2][2]) {
    const T one(1);
    g[0][0][0] = dL * (one - a.x) * (one - a.y) * (one - a.z);
    g[0][0][1] = dL * (a.x) * (one - a.y) * (one - a.z);
    g[0][1][0] = dL * (one - a.x) * (a.y) * (one - a.z);
    g[0][1][1] = dL * (a.x) * (a.y) * (one - a.z);
    g[1][0][0] = dL * (one - a.x) * (one - a.y) * (a.z);
    g[1][0][1] = dL * (a.x) * (one - a.y) * (a.z);
    g[1][1][0] = dL * (one - a.x) * (a.y) * (a.z);
    g[1][1][1] = dL * (a.x) * (a.y) * (a.z);
}

// ---------------------------------------------------------------------------
// include/vr_transmittance_DDA.h:1-59 (fw) and :62-156 (bw).
// exact == false: the reference's per-cell midpoint rule (its "TODO" at :41).
// exact == true (extension): two-point Gauss-Legendre per cell, which is exact
// for the cubic that a trilinear field restricted to a segment is.
// ---------------------------------------------------------------------------
template <typename T> struct DDA {
    const Scene<T>& S;
    V3<T> x, w, bmin, box_size, cell_size, alpha_inc, corner, alpha, vn, vm;
    int dim[3], cell[3], side[3];
    T d;
    bool valid;

    DDA(const Scene<T>& sc, V3<T> x0, V3<T> w0) : S(sc), x(x0), w(w0) {
        valid = false;
        T tMin, tMax;
        if (!S.boundary(x, w, tMin, tMax)) return;
        T gMin, gMax;
        V3<T> gbmin = V3<T>::load(S.s.bmin), gbmax = V3<T>::load(S.s.bmax);
        if (!intersect_ray_box(x, w, gbmin, gbmax, gMin, gMax)) return;
        tMin = vmax(tMin, gMin);
        tMax = vmin(tMax, gMax);
        if (tMax <= tMin) return;
        valid = true;
        x = x + w * tMin;
        d = tMax - tMin;
        bmin = gbmin;
        box_size = gbmax - gbmin;
        dim[0] = S.s.sigma.W - 1; dim[1] = S.s.sigma.H - 1; dim[2] = S.s.sigma.D - 1;
        V3<T> fdim((T)dim[0], (T)dim[1], (T)dim[2]);
        cell_size = box_size / fdim;
        V3<T> cc = (x - bmin) * fdim / box_size;
        for (int i = 0; i < 3; ++i) cell[i] = std::min(std::max((int)cc[i], 0), dim[i] - 1);
        V3<T> aw(std::abs(w.x), std::abs(w.y), std::abs(w.z));
        V3<T> den(vmax(T(0.000001), aw.x), vmax(T(0.000001), aw.y), vmax(T(0.000001), aw.z));
        alpha_inc = cell_size / den;
        for (int i = 0; i < 3; ++i) side[i] = w[i] > T(0) ? 1 : (w[i] < T(0) ? -1 : 0);
        corner = (V3<T>((T)cell[0], (T)cell[1], (T)cell[2]) + V3<T>((T)side[0], (T)side[1], (T)side[2]) * T(0.5) +
                  V3<T>(T(0.5))) * cell_size + bmin;
        V3<T> cd = corner - x;
        alpha = V3<T>(std::abs(cd.x), std::abs(cd.y), std::abs(cd.z)) / den;
        vn = (x - bmin) * fdim / box_size;
        vm = w * fdim / box_size;
    }
    void reset_march() {
        V3<T> fdim((T)dim[0], (T)dim[1], (T)dim[2]);
        V3<T> cc = (x - bmin) * fdim / box_size;
        for (int i = 0; i < 3; ++i) cell[i] = std::min(std::max((int)cc[i], 0), dim[i] - 1);
        V3<T> aw(std::abs(w.x), std::abs(w.y), std::abs(w.z));
        V3<T> den(vmax(T(0.000001), aw.x), vmax(T(0.000001), aw.y), vmax(T(0.000001), aw.z));
        V3<T> cd = corner - x;
        alpha = V3<T>(std::abs(cd.x), std::abs(cd.y), std::abs(cd.z)) / den;
    }
    void load_cell(T s[2][2][2]) const {  // vr_sigma_grid.h:9-16
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) s[dz][dy][dx] = S.sigma_at(cell[0] + dx, cell[1] + dy, cell[2] + dz);
    }
    V3<T> ialpha(T t) const {
        return (vm * t + vn) - V3<T>((T)cell[0], (T)cell[1], (T)cell[2]);
    }
    void step() {  // vr_transmittance_DDA.h:48-55
        int inc[3] = {alpha.x <= alpha.y && alpha.x <= alpha.z, alpha.x > alpha.y && alpha.y <= alpha.z,
                      alpha.x > alpha.z && alpha.y > alpha.z};
        for (int i = 0; i < 3; ++i) {
            alpha[i] = alpha[i] + T(inc[i]) * alpha_inc[i];
            cell[i] += inc[i] * side[i];
        }
    }

    static constexpr double GL = 0.28867513459481288225;  // 1/(2 sqrt 3)

    // The reference stops 1e-4 short of the exit (vr_transmittance_DDA.h:38);
    // the exact mode (an extension) integrates the whole segment.
    T tau(bool exact, int64_t* steps) {
        T acc = 0, ct = 0;
        T s[2][2][2];
        const T stop = exact ? d : d - T(0.0001);
        while (ct < stop) {
            T nt = vmin(d, vmin(alpha.x, vmin(alpha.y, alpha.z)));
            load_cell(s);
            T dt = nt - ct;
            if (!exact) {
                T cell_t = mix(ct, nt, T(0.5));
                acc += interpolated_sigma(ialpha(cell_t), s) * dt;
            } else {
                T mid = mix(ct, nt, T(0.5)), h = dt * T(GL);
                acc += (interpolated_sigma(ialpha(mid - h), s) + interpolated_sigma(ialpha(mid + h), s)) * (dt * T(0.5));
            }
            if (steps) ++*steps;
            ct = nt;
            step();
        }
        return acc;
    }
    void tau_bw(bool exact, T dL_dtau) {
        T ct = 0;
        T g[2][2][2], g2[2][2][2];
        const T stop = exact ? d : d - T(0.0001);
        while (ct < stop) {
            T nt = vmin(d, vmin(alpha.x, vmin(alpha.y, alpha.z)));
            T dt = nt - ct;
            if (!exact) {
                T cell_t = mix(ct, nt, T(0.5));
                interpolated_sigma_bw(ialpha(cell_t), dL_dtau * dt, g);
            } else {
                T mid = mix(ct, nt, T(0.5)), h = dt * T(GL);
                interpolated_sigma_bw(ialpha(mid - h), dL_dtau * dt * T(0.5), g);
                interpolated_sigma_bw(ialpha(mid + h), dL_dtau * dt * T(0.5), g2);
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b)
                        for (int c = 0; c < 2; ++c) g[a][b][c] += g2[a][b][c];
            }
            for (int dz = 0; dz < 2; ++dz)  // vr_sigma_grid.h:65-75 update_cell_gradients
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx)
                        S.sigma_at_bw(cell[0] + dx, cell[1] + dy, cell[2] + dz, g[dz][dy][dx]);
            ct = nt;
            step();
        }
    }
};

// include/vr_transmittance_GRT.h:1-83 (delta == false) and
// include/vr_transmittance_GDT.h:1-84 (delta == true): the DDA walk of the
// grid's cells; per cell the eight corner values give a majorant and a
// minorant, the minorant part is integrated in closed form and the residual
// sigma - minorant is tracked against majorant - minorant.  Forward only (the
// reference's maps have no backward).
template <typename T>
T transmittance_grid_tracking(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, bool delta, int64_t* steps) {
    DDA<T> dda(S, x, w);
    if (!dda.valid) return T(1);
    T Tr = T(1), ct = T(0);
    T s[2][2][2];
    while (ct < dda.d - T(0.0001)) {
        T nt = vmin(dda.d, vmin(dda.alpha.x, vmin(dda.alpha.y, dda.alpha.z)));
        dda.load_cell(s);
        T mx = s[0][0][0], mn = s[0][0][0];
        for (int k = 1; k < 8; ++k) {
            const T v = s[k >> 2][(k >> 1) & 1][k & 1];
            mx = std::max(mx, v);
            mn = std::min(mn, v);
        }
        if (steps) ++*steps;
        Tr *= std::exp(-mn * (nt - ct));
        const T rm = vmax(T(0.000001), mx - mn);
        T cell_t = ct;
        while (true) {
            const T dt = -std::log(T(1) - (T)rng.uniform()) / rm;
            if (cell_t + dt > nt) break;
            cell_t += dt;
            const T sv = interpolated_sigma(dda.ialpha(cell_t), s);
            const T Pc = (sv - mn) / rm;
            if (steps) ++*steps;
            if (delta) {
                if ((T)rng.uniform() < Pc) return T(0);
            } else {
                Tr *= (T(1) - Pc);
            }
        }
        ct = nt;
        dda.step();
    }
    return Tr;
}

template <typename T> T transmittance_DDA(const Scene<T>& S, V3<T> x, V3<T> w, bool exact, int64_t* steps) {
    DDA<T> dda(S, x, w);
    if (!dda.valid) return T(1);
    return std::exp(-dda.tau(exact, steps));
}
template <typename T> void transmittance_DDA_bw(const Scene<T>& S, V3<T> x, V3<T> w, bool exact, T dL_dT) {
    if (dL_dT == T(0)) return;
    if (!S.s.sigma.grad) return;  // include/maps/transmittance_dda.h:21 sigma_grid_has_grad
    DDA<T> dda(S, x, w);
    if (!dda.valid) return;
    T tau = dda.tau(exact, nullptr);
    T Tr = std::exp(-tau);
    T dL_dtau = -dL_dT * Tr;
    dda.reset_march();
    dda.tau_bw(exact, dL_dtau);
}

// ---------------------------------------------------------------------------
// include/vr_transmittance_RT.h:1-49 ratio tracking.  The branch marked
// "grid crossing" restarts at a majorant-brick face without a collision; it
// is reachable only with the majorant grid (the reference's majorant distance
// is 1e6, beyond any segment).
// ---------------------------------------------------------------------------
template <typename T> T transmittance_RT(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, int64_t* steps) {
    T Tr = 1;
    T tMin, tMax;
    if (!S.boundary(x, w, tMin, tMax)) return Tr;
    x += w * tMin;
    T d = tMax - tMin;
    for (Flight<T> ff; ff.it < (1 << 24); ++ff.it) {
        T md;
        T maj = vmax(T(0.0000001), ff.bk.query(S.s, x, w, md));
        T t = ff.sample(rng) / maj;
        if (steps) ++*steps;
        if (md < d && t > md) { x += w * md; d -= md; ff.cross(maj, md); ff.bk.advance(S.s); continue; }  // grid crossing
        ff.used();
        T dt = vmin(t, vmin(d, md));
        ff.bk.move(dt);
        x += w * dt;
        d -= dt;
        if (d <= T(0.0000001)) return Tr;
        Tr *= (T(1) - S.sigma(x) / maj);
        if (Tr < T(0.01)) {
            if ((T)rng.uniform() < T(1) - Tr) return T(0);
            Tr = T(1);
        }
    }
    return Tr;
}

// include/vr_transmittance_RT.h:51-141 (two passes from the same draws)
template <typename T> void transmittance_RT_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T dL_dT) {
    if (dL_dT == T(0)) return;
    T tMin, tMax;
    if (!S.boundary(x, w, tMin, tMax)) return;
    const T EPS = T(0.0000001);
    T Tr = 1;
    x += w * tMin;
    T d = tMax - tMin;
    V3<T> ini_x = x;
    T ini_d = d;
    Rng before = rng;
    for (Flight<T> ff; ff.it < (1 << 24); ++ff.it) {
        T md;
        T maj = vmax(EPS, ff.bk.query(S.s, x, w, md) + T(0.1));
        T t = ff.sample(rng) / maj;
        if (md < d && t > md) { x += w * md; d -= md; ff.cross(maj, md); ff.bk.advance(S.s); continue; }  // grid crossing
        ff.used();
        T dt = vmin(t, vmin(d, md));
        ff.bk.move(dt);
        x += w * dt;
        d -= dt;
        if (d <= EPS) break;
        Tr *= (T(1) - S.sigma(x) / maj);
        if (Tr < T(0.1)) {
            if ((T)rng.uniform() < T(1) - Tr) return;
            Tr = T(1);
        }
    }
    T out_T = Tr;
    Tr = 1;
    rng = before;
    x = ini_x;
    d = ini_d;
    for (Flight<T> ff; ff.it < (1 << 24); ++ff.it) {
        T md;
        T maj = vmax(EPS, ff.bk.query(S.s, x, w, md) + T(0.1));
        T t = ff.sample(rng) / maj;
        if (md < d && t > md) { x += w * md; d -= md; ff.cross(maj, md); ff.bk.advance(S.s); continue; }  // grid crossing
        ff.used();
        T dt = vmin(t, vmin(d, md));
        ff.bk.move(dt);
        x += w * dt;
        d -= dt;
        if (d <= EPS) break;
        T r = (T(1) - S.sigma(x) / maj);
        Tr *= r;
        T dL_dsigma = -out_T * dL_dT / maj / r;
        S.sigma_bw(x, dL_dsigma);
        if (Tr < T(0.1)) {
            rng.advance();
            Tr = T(1);
        }
    }
}

// include/vr_transmittance_DT.h:1-28
template <typename T> T transmittance_DT(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, int64_t* steps) {
    T tMin, tMax;
    if (!S.boundary(x, w, tMin, tMax)) return T(1);
    x += w * tMin;
    T d = tMax - tMin;
    for (Flight<T> ff; ff.it < (1 << 24); ++ff.it) {
        T md;
        T maj = vmax(T(0.0000001), ff.bk.query(S.s, x, w, md));
        T dt = ff.sample(rng) / maj;
        T t = vmin(md, dt);
        if (steps) ++*steps;
        x += w * t;
        d -= t;
        // the end test precedes the brick-crossing restart (the reference's
        // order, which the constant majorant never distinguishes)
        if (d <= T(0.0000001)) return T(1);
        if (dt > md) { ff.cross(maj, md); ff.bk.advance(S.s); continue; }
        ff.used();
        ff.bk.move(t);
        if ((T)rng.uniform() < S.sigma(x) / maj) return T(0);
    }
    return T(1);
}

// include/vr_transmittance_DT.h:30-90
template <typename T> void transmittance_DT_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T dL_dT) {
    if (dL_dT == T(0)) return;
    T tMin, tMax;
    if (!S.boundary(x, w, tMin, tMax)) return;
    x += w * tMin;
    T d = tMax - tMin;
    V3<T> ini_x = x;
    T ini_d = d;
    Rng before = rng;
    for (Flight<T> ff; ff.it < (1 << 24); ++ff.it) {
        T md;
        T maj = vmax(T(0.0000001), ff.bk.query(S.s, x, w, md) + T(0.1));
        T dt = ff.sample(rng) / maj;
        T t = vmin(md, dt);
        x += w * t;
        d -= t;
        if (d <= T(0.0000001)) break;
        if (dt > md) { ff.cross(maj, md); ff.bk.advance(S.s); continue; }
        ff.used();
        ff.bk.move(t);
        if ((T)rng.uniform() < S.sigma(x) / maj) return;
    }
    x = ini_x;
    d = ini_d;
    rng = before;
    for (Flight<T> ff; ff.it < (1 << 24); ++ff.it) {
        T md;
        T maj = vmax(T(0.0000001), ff.bk.query(S.s, x, w, md) + T(0.1));
        T dt = ff.sample(rng) / maj;
        T t = vmin(md, dt);
        x += w * t;
        d -= t;
        if (d <= T(0.0000001)) break;
        if (dt > md) { ff.cross(maj, md); ff.bk.advance(S.s); continue; }
        ff.used();
        ff.bk.move(t);
        rng.advance();
        T Pc = S.sigma(x) / maj;
        T dL_dsigma = -dL_dT / maj / (T(1) - Pc);
        S.sigma_bw(x, dL_dsigma);
    }
}

// include/vr_transmittance.h dispatch over the lowered transmittance map
template <typename T> T transmittance(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, int64_t* steps) {
    Rng sr = rng.fork();
    switch (S.s.transmittance_mode) {
        case 0: return transmittance_RT(S, sr, x, w, steps);
        case 1: return transmittance_DT(S, sr, x, w, steps);
        case 2: return transmittance_DDA(S, x, w, false, steps);
        case 3: return transmittance_DDA(S, x, w, true, steps);
        case 4: return transmittance_grid_tracking(S, sr, x, w, false, steps);
        default: return transmittance_grid_tracking(S, sr, x, w, true, steps);
    }
}
template <typename T> void transmittance_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T dL_dT) {
    Rng sr = rng.fork();
    switch (S.s.transmittance_mode) {
        case 0: transmittance_RT_bw(S, sr, x, w, dL_dT); break;
        case 1: transmittance_DT_bw(S, sr, x, w, dL_dT); break;
        case 2: transmittance_DDA_bw(S, x, w, false, dL_dT); break;
        case 3: transmittance_DDA_bw(S, x, w, true, dL_dT); break;
        default: break;  // GRT / GDT: no backward (the reference's maps define none)
    }
}

// ---------------------------------------------------------------------------
// Directions: include/randoms.h:144-162 createOrthoBasis / randomDirection,
// include/scattering_AD.h:4-52 hg_phase_sample / hg_phase_eval.
// ---------------------------------------------------------------------------
template <typename T> void ortho_basis(V3<T> N, V3<T>& t, V3<T>& b) {
    T sign = N.z >= T(0) ? T(1) : T(-1);
    T a = T(-1) / (sign + N.z);
    T bb = N.x * N.y * a;
    t = V3<T>(T(1) + sign * N.x * N.x * a, sign * bb, -sign * N.x);
    b = V3<T>(bb, sign + N.y * N.y * a, -N.y);
}
template <typename T> V3<T> random_direction(Rng& rng, V3<T> D) {
    T r1 = (T)rng.uniform();
    T r2 = (T)rng.uniform() * T(2) - T(1);
    T sq = r2 * r2;
    T ang = K<T>::two_pi * r1;
    T st = std::sqrt(vmax(T(0), T(1) - sq));
    T x = std::cos(ang) * st, y = std::sin(ang) * st, z = r2;
    V3<T> t0, t1;
    ortho_basis(D, t0, t1);
    return t0 * x + t1 * y + D * z;
}
template <typename T> V3<T> hg_phase_sample(Rng& rng, V3<T> w_in, T g) {
    T phi = (T)rng.uniform() * T(2) * K<T>::pi;
    T xi = (T)rng.uniform();
    T g2 = g * g;
    T omg2 = T(1) - g2, opg2 = T(1) + g2;
    T o2g = T(0.5) / g;
    T t = omg2 / (T(1) - g + T(2) * g * xi);
    T inv = o2g * (opg2 - t * t);
    T ct = std::abs(g) < T(0.001) ? T(2) * xi - T(1) : inv;
    T st = std::sqrt(vmax(T(0), T(1) - ct * ct));
    V3<T> t0, t1;
    ortho_basis(w_in, t0, t1);
    return st * std::sin(phi) * t0 + st * std::cos(phi) * t1 + ct * w_in;
}
template <typename T> T hg_phase_eval(T c, T g) {
    if (std::abs(g) < T(0.001)) return T(0.25) / K<T>::pi;
    T g2 = g * g;
    return T(0.25) / K<T>::pi * (T(1) - g2) / std::pow(T(1) + g2 - T(2) * g * c, T(1.5));
}

// include/vr_phase.h over HGPhase (_maps.py:4436-4460, mode 1) or pure HG (mode 0)
template <typename T> T phase(const Scene<T>& S, V3<T> w, V3<T> wo) {
    T g = (T)S.s.phase_g;
    T c = dot(w, wo);
    if (S.s.phase_mode == 1) return mix(hg_phase_eval(c, g), hg_phase_eval(c, g / T(5)), T(0.2));
    return hg_phase_eval(c, g);
}
// include/vr_phase_sampler.h over VHGPhaseSampler (_maps.py:4463-4484, mode 1) or pure HG (mode 0)
template <typename T> T phase_sampler(const Scene<T>& S, Rng& rng, V3<T> w, V3<T>& wo) {
    T g = (T)S.s.phase_g;
    if (S.s.phase_mode == 1) {
        if ((T)rng.uniform() < T(0.8)) g = g / T(5);
    }
    wo = hg_phase_sample(rng, w, g);
    return T(1);
}
// include/vr_environment_sampler.h over _functionsampler(UniformDirectionSampler, const env)
// (_maps.py:2552-2585, include/maps/uniform_direction_sampler.h:1-5)
// or over XRQuadtreeRandomDirection (_maps.py:2494-2549): a pixel drawn down
// the probability quadtree with one uniform, then a direction uniform in its
// solid angle (include/randoms.h:186-199 randomDirection); weight = pixel
// solid angle / p.
template <typename T> V3<T> environment_sampler(const Scene<T>& S, Rng& rng, V3<T>& wo) {
    if (S.s.env_sampler == 0) {
        wo = random_direction(rng, V3<T>(T(0), T(1), T(0)));
        T weight = T(4) * K<T>::pi;
        return S.environment(wo) * weight;
    }
    float sel = rng.uniform();
    int64_t node = 0;
    float p0x = 0.0f, p0y = 0.0f, p1x = 1.0f, p1y = 1.0f, prob = 1.0f;
    for (int i = 0; i < S.s.env_levels; ++i) {
        const float* d = S.s.env_quadtree + node * 4;
        int child = 3;
        prob = d[3];
        for (int c = 0; c < 3; ++c) {
            if (sel < d[c]) {
                child = c;
                prob = d[c];
                break;
            }
            sel -= d[c];
        }
        const float xmed = (p1x + p0x) / 2.0f, ymed = (p1y + p0y) / 2.0f;
        if (child % 2 == 0) p1x = xmed; else p0x = xmed;
        if (child / 2 == 0) p1y = ymed; else p0y = ymed;
        node = node * 4 + 1 + child;
    }
    const T pi = K<T>::pi;
    const T pixel_area = T(2) * pi * (std::cos((T)p0y * pi) - std::cos((T)p1y * pi)) / T(1 << S.s.env_levels);
    const T weight = pixel_area / std::max(T(0.000000001), (T)prob);
    const T a0 = ((T)p0x * T(2) - T(1)) * pi, a1 = ((T)p1x * T(2) - T(1)) * pi, b0 = (T)p0y * pi, b1 = (T)p1y * pi;
    const T r1 = (T)rng.uniform() * (a1 - a0) + a0;
    const T r2 = std::cos(b0) - (T)rng.uniform() * (std::cos(b0) - std::cos(b1));
    const T sq = std::sqrt(std::max(T(0), T(1) - r2 * r2));
    wo = V3<T>(std::sin(r1) * sq, r2, std::cos(r1) * sq);
    return S.environment(wo) * weight;
}

// ---------------------------------------------------------------------------
// include/vr_path_integrator_NEE.h:1-66, plus the extensions: a directional
// light sampled after the environment at every real collision, and an
// optional bounce cap (0 keeps the reference's uncapped loop).
// ---------------------------------------------------------------------------
// Hooks of the radiance-cache forms (no reference counterpart).  cut >= 0: a
// path reaching its (cut+1)-th real collision records (x, w, W) there and stops
// (the cache adds W * L(x, w) later).  rec > 0: the first rec collisions record
// (x, w, W, R so far) so the caller can form the in-scattered radiance targets
// (R_final - R_k) / W_k.
template <typename T> struct PathHooks {
    int cut = -1, rec = 0;
    bool queried = false;
    V3<T> qx, qw, qW;
    int nrec = 0;
    V3<T> rx[8], rw[8], rW[8], rR[8];
};

template <typename T>
V3<T> path_integrator_NEE(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, bool only_scatters, Counters& cnt,
                          PathHooks<T>* hk = nullptr) {
    T tMin, tMax;
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    T d = tMax - tMin;
    V3<T> R(T(0)), W(T(1));
    if (!only_scatters) R += transmittance(S, rng, x, w, &cnt.steps) * S.environment(w);
    const T EPS = T(0.00001);
    int bounces = 0;
    const V3<T> sun_dir = V3<T>::load(S.s.sun_dir), sun_L = V3<T>::load(S.s.sun_radiance);
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = vmax(EPS, ff.bk.query(S.s, x, w, md));
        T t = ff.sample(rng) / m;
        ++cnt.steps;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        T Pc = s / m;
        if ((T)rng.uniform() >= Pc) { d -= t; continue; }
        ++cnt.vertices;
        if (hk && hk->cut >= 0 && bounces == hk->cut) {
            hk->queried = true;
            hk->qx = x; hk->qw = w; hk->qW = W;
            return R;
        }
        if (hk && bounces < hk->rec) {
            hk->rx[bounces] = x; hk->rw[bounces] = w; hk->rW[bounces] = W; hk->rR[bounces] = R;
            hk->nrec = bounces + 1;
        }
        V3<T> sa = S.albedo(x);
        V3<T> em = S.emission();
        R += W * (V3<T>(T(1)) - sa) * em;
        W *= sa;
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        T T_nee = transmittance(S, rng, x, wnee, &cnt.steps);
        R += W * T_nee * env * phase(S, w, wnee);
        if (S.s.has_sun) {
            T T_sun = transmittance(S, rng, x, sun_dir, &cnt.steps);
            R += W * T_sun * sun_L * phase(S, w, sun_dir);
        }
        ++bounces;
        if (S.s.max_bounces > 0 && bounces >= S.s.max_bounces) return R;
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        W *= rho;
        if (all_less(W, EPS)) return R;
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
    }
    return R;
}

// include/vr_path_integrator_DT.h:7-57 (no NEE; escape term W*env)
template <typename T> V3<T> path_integrator_DT(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, Counters& cnt) {
    T tMin, tMax;
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    T d = tMax - tMin;
    V3<T> R(T(0)), W(T(1));
    int bounces = 0;
    for (Flight<T> ff; d > T(0.00000001);) {
        T md;
        T m = vmax(T(0.00000001), ff.bk.query(S.s, x, w, md));
        T t = ff.sample(rng) / m;
        ++cnt.steps;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        T Pc = s / m;
        if ((T)rng.uniform() >= Pc) { d -= t; continue; }
        ++cnt.vertices;
        V3<T> sa = S.albedo(x);
        V3<T> em = S.emission();
        R += W * (V3<T>(T(1)) - sa) * em;
        W *= sa;
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        W *= rho;
        if (all_less(W, T(0.0000001))) return R;
        if (S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces) return R;
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
    }
    return W * S.environment(w) + R;
}

// include/vr_path_integrator_DT.h:59-235 path_integrator_DT_bw
template <typename T> void path_integrator_DT_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T eps, V3<T> dL_dR) {
    Rng before_path = rng;
    V3<T> ini_x = x, ini_w = w;
    T tMin, tMax;
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    T d = tMax - tMin;
    const T EPS = T(0.00000001);
    V3<T> W(T(1));
    T null_W = 1;
    int bounces = 0;
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = vmax(EPS, ff.bk.query(S.s, x, w, md) + T(2) * eps);
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        T Pc = (s + eps) / m;
        if ((T)rng.uniform() >= Pc) { d -= t; W *= (T(1) - s / m) / (T(1) - Pc); continue; }
        if (s == T(0)) {
            if (null_W == T(0)) { W = V3<T>(T(0)); break; }
            null_W = 0;
        } else
            W *= (s / m) / Pc;
        V3<T> sa = S.albedo(x);
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        W *= sa * rho;
        if (all_less(W, EPS)) { W = V3<T>(T(0)); break; }
        if (S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces) { W = V3<T>(T(0)); break; }
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
    }
    V3<T> env = S.environment(w);
    V3<T> dL_dW = dL_dR * env;
    rng = before_path;
    x = ini_x;
    w = ini_w;
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    d = tMax - tMin;
    V3<T> W_out = W;
    W = V3<T>(T(1));
    bounces = 0;
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = vmax(EPS, ff.bk.query(S.s, x, w, md) + T(2) * eps);
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        T Pc = (s + eps) / m;
        if ((T)rng.uniform() >= Pc) {
            T dL_dsigma = dot(dL_dW, -W_out * null_W / m / (T(1) - s / m));
            S.sigma_bw(x, dL_dsigma);
            W *= (T(1) - s / m) / (T(1) - Pc);
            d -= t;
            continue;
        }
        {
            T dL_dsigma = dot(dL_dW, s == T(0) ? W_out : W_out * null_W / s);
            S.sigma_bw(x, dL_dsigma);
        }
        W *= s / m / Pc;
        if (s == T(0)) break;
        V3<T> sa = S.albedo(x);
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        W *= sa;
        W *= rho;
        if (all_less(W, EPS)) return;
        if (S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces) return;
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
    }
}

// include/vr_path_integrator_NEE_DS.h:6-206 path_integrator_NEE_DS_bw.  With
// ds_compat == 1 the replay uses the reference's majorant (x1.2 + 2 eps) that
// differs from its primal pass (+ 2 eps + 0.1); with 0 both passes share the
// primal majorant so that the replay retraces the primal path.
template <typename T> void path_integrator_NEE_DS_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T eps, V3<T> dL_dR) {
    Rng before_path = rng;
    V3<T> ini_x = x, ini_w = w;
    T tMin, tMax;
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    T d = tMax - tMin;
    V3<T> R(T(0)), R_after_sp(T(0)), W(T(1));
    T null_W = 1;
    const T EPS = T(0.00000001);
    bool scattered = false;
    int bounces = 0;
    const V3<T> sun_dir = V3<T>::load(S.s.sun_dir), sun_L = V3<T>::load(S.s.sun_radiance);
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = vmax(EPS, ff.bk.query(S.s, x, w, md) + T(2) * eps + T(0.1));
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        T Pc = (s + eps) / m;
        if ((T)rng.uniform() >= Pc) { d -= t; W *= (T(1) - s / m) / (T(1) - Pc); continue; }
        scattered = true;
        if (s < EPS) {
            if (null_W < EPS) { W = V3<T>(T(0)); break; }
            null_W = 0;
        } else
            W *= (s / m) / Pc;
        V3<T> em = S.emission();
        V3<T> sa = S.albedo(x);
        V3<T> added_R = W * (V3<T>(T(1)) - sa) * em;
        W *= sa;
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        T T_nee = transmittance(S, rng, x, wnee, nullptr);
        T ph_nee = phase(S, w, wnee);
        added_R += W * T_nee * env * ph_nee;
        if (S.s.has_sun) {
            T T_sun = transmittance(S, rng, x, sun_dir, nullptr);
            added_R += W * T_sun * sun_L * phase(S, w, sun_dir);
        }
        if (null_W < EPS) R_after_sp += added_R;
        else R += added_R;
        if (S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces) { W = V3<T>(T(0)); break; }
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        W *= rho;
        if (all_less(W, EPS)) { W = V3<T>(T(0)); break; }
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
    }
    if (!scattered) R += S.environment(w) * W;

    rng = before_path;
    x = ini_x;
    w = ini_w;
    W = V3<T>(T(1));
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    d = tMax - tMin;
    bounces = 0;
    for (Flight<T> ff; d > EPS;) {
        T md;
        T mj = ff.bk.query(S.s, x, w, md);
        T m = S.s.ds_compat ? vmax(EPS, mj * T(1.2) + T(2) * eps) : vmax(EPS, mj + T(2) * eps + T(0.1));
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        T Pc = (s + eps) / m;
        T dL_dsigma;
        if ((T)rng.uniform() >= Pc) {
            dL_dsigma = dot(dL_dR, -R / m / (T(1) - s / m));
            S.sigma_bw(x, dL_dsigma);
            W *= (T(1) - s / m) / (T(1) - Pc);
            d -= t;
            continue;
        }
        dL_dsigma = dot(dL_dR, s < EPS ? R_after_sp / eps : R / s);
        S.sigma_bw(x, dL_dsigma);
        W *= s / m / Pc;
        if (s < EPS) return;
        V3<T> em = S.emission();
        V3<T> sa = S.albedo(x);
        V3<T> dL_dsa = dL_dR * W * T(-1) * em;
        R -= W * (V3<T>(T(1)) - sa) * em;
        dL_dsa += dL_dR * R / V3<T>(vmax(EPS, sa.x), vmax(EPS, sa.y), vmax(EPS, sa.z));
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        Rng before_transmittance = rng;
        T T_nee = transmittance(S, rng, x, wnee, nullptr);
        T ph_nee = phase(S, w, wnee);
        Rng before_sun = rng;
        T T_sun = 0, ph_sun = 0;
        if (S.s.has_sun) {
            T_sun = transmittance(S, rng, x, sun_dir, nullptr);
            ph_sun = phase(S, w, sun_dir);
        }
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        Rng before_next = rng;
        W *= sa;
        T dL_dTnee = dot(dL_dR, W * env * ph_nee);
        R -= W * T_nee * env * ph_nee;
        T dL_dTsun = 0;
        if (S.s.has_sun) {
            dL_dTsun = dot(dL_dR, W * sun_L * ph_sun);
            R -= W * T_sun * sun_L * ph_sun;
        }
        S.albedo_bw(x, dL_dsa);
        rng = before_transmittance;
        transmittance_bw(S, rng, x, wnee, dL_dTnee);
        if (S.s.has_sun) {
            rng = before_sun;
            transmittance_bw(S, rng, x, sun_dir, dL_dTsun);
        }
        rng = before_next;
        if (S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces) return;
        W *= rho;
        if (all_less(W, EPS)) return;
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
    }
}

// include/vr_path_integrator_NEE_DRT.h:8-60 sample_transmittance_position.
// The majorant is queried at the current sample point x + w t (the reference
// queries it at x, which is the same for its constant majorant).
template <typename T>
T sample_transmittance_position(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T d, T& sample_t, T& weight_t) {
    T Tr = 1, t = 0, res_t = 0, res_dt = 0, C = 0;
    const T EPS = T(0.0000001);
    for (Flight<T> ff; ff.it < (1 << 24); ++ff.it) {
        T md;
        T m = vmax(EPS, S.majorant(x + w * t, w, md));
        T dt = vmin(-std::log(T(1) - (T)rng.uniform()) / m, vmin(md, d - t));
        T w_step = Tr * dt;
        C += w_step;
        if ((T)rng.uniform() < w_step / C) { res_t = t; res_dt = dt; }
        t += dt;
        if (dt >= md - EPS) continue;
        if (t >= d - EPS) break;
        Tr *= T(1) - S.sigma(x + w * t) / m;
    }
    weight_t = C;
    sample_t = res_t + (T)rng.uniform() * res_dt;
    return Tr;
}

// include/vr_path_integrator_NEE_DRT.h:62-270 path_integrator_NEE_DRT_bw.
// The branch seed becomes Philox stream 1 of the same path.
template <typename T> void path_integrator_NEE_DRT_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, V3<T> dL_dR) {
    T tMin, tMax;
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    T d = tMax - tMin;
    if (d <= T(0)) return;
    Rng sec = rng;  // the branch seed (BRANCH_SEED(secondary_seed)) is stream 1
    sec.stream = rng.stream + 1;
    sec.n = 0;
    sec.ntr = 0;
    Counters dummy;
    T direct_T = transmittance(S, rng, x, w, nullptr);
    V3<T> direct_env = S.environment(w);
    T dL_ddT = dot(dL_dR, direct_env);
    transmittance_bw(S, sec, x, w, dL_ddT);
    V3<T> R(T(0)), W(T(1));
    V3<T> res_x = x, res_w = w, res_W = W;
    T res_P = 3, total_weight = 3;
    V3<T> ini_x = x, ini_w = w;
    T ini_d = d;
    const T EPS = T(0.00000001);
    const V3<T> sun_dir = V3<T>::load(S.s.sun_dir), sun_L = V3<T>::load(S.s.sun_radiance);
    Rng before_path = rng;
    int bounces = 0;
    (void)direct_T;
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = ff.bk.query(S.s, x, w, md) * T(1.05) + T(0.1);
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        T Pc = s / m;
        if ((T)rng.uniform() >= Pc) { d -= t; continue; }
        V3<T> sa = S.albedo(x);
        W *= sa;
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        T T_nee = transmittance(S, rng, x, wnee, nullptr);
        T ph_nee = phase(S, w, wnee);
        R += W * T_nee * env * ph_nee;
        if (S.s.has_sun) {
            T T_sun = transmittance(S, rng, x, sun_dir, nullptr);
            R += W * T_sun * sun_L * phase(S, w, sun_dir);
        }
        bool capped = S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces;
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        W *= rho;
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
        T current_P = W.x + W.y + W.z;
        total_weight += current_P;
        if ((T)rng.uniform() < current_P / total_weight) {
            res_P = current_P; res_W = W; res_x = x; res_w = w;
        }
        if (all_less(W, EPS) || capped) break;
    }
    W = V3<T>(T(1));
    x = ini_x;
    w = ini_w;
    d = ini_d;
    rng = before_path;
    bounces = 0;
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = ff.bk.query(S.s, x, w, md) * T(1.05) + T(0.1);
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        T Pc = s / m;
        T dL_dsigma;
        if ((T)rng.uniform() >= Pc) {
            dL_dsigma = dot(dL_dR, -R / m / (T(1) - s / m));
            S.sigma_bw(x, dL_dsigma);
            d -= t;
            continue;
        }
        T mis_weight_Ts = s * s / (T(1) + s * s);
        dL_dsigma = dot(dL_dR, mis_weight_Ts * R / s);
        V3<T> sa = S.albedo(x);
        W *= sa;
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        T T_nee = transmittance(S, rng, x, wnee, nullptr);
        T ph_nee = phase(S, w, wnee);
        T T_sun = 0, ph_sun = 0;
        if (S.s.has_sun) {
            T_sun = transmittance(S, rng, x, sun_dir, nullptr);
            ph_sun = phase(S, w, sun_dir);
        }
        bool capped = S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces;
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        T dL_dTnee = dot(dL_dR, W * env * ph_nee);
        R -= W * T_nee * env * ph_nee;
        T dL_dTsun = 0;
        if (S.s.has_sun) {
            dL_dTsun = dot(dL_dR, W * sun_L * ph_sun);
            R -= W * T_sun * sun_L * ph_sun;
        }
        S.sigma_bw(x, dL_dsigma);
        transmittance_bw(S, sec, x, wnee, dL_dTnee);
        if (S.s.has_sun) transmittance_bw(S, sec, x, sun_dir, dL_dTsun);
        W *= rho;
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
        rng.advance();
        if (all_less(W, EPS) || capped) break;
    }
    S.boundary(res_x, res_w, tMin, d);
    T s_t, weight_t;
    sample_transmittance_position(S, rng, res_x, res_w, d, s_t, weight_t);
    V3<T> xs = res_x + res_w * s_t;
    V3<T> ls_dir;
    V3<T> Ls_env = environment_sampler(S, rng, ls_dir);
    V3<T> Ls = transmittance(S, rng, xs, ls_dir, nullptr) * Ls_env * phase(S, res_w, ls_dir);
    if (S.s.has_sun) Ls += transmittance(S, rng, xs, sun_dir, nullptr) * sun_L * phase(S, res_w, sun_dir);
    V3<T> ws;
    T rho_s = phase_sampler(S, rng, res_w, ws);
    Ls += rho_s * path_integrator_NEE(S, rng, xs, ws, true, dummy);
    Ls *= res_W * weight_t * S.albedo(xs);
    T sigma_xs = S.sigma(xs);
    T mis_weight_T = T(1) / (T(1) + sigma_xs * sigma_xs);
    T dL_dsc = dot(dL_dR, Ls) * mis_weight_T * total_weight / res_P;
    S.sigma_bw(xs, dL_dsc);
}

// include/vr_path_integrator_NEE_DRTQ.h:45-55 in_scattering, plus the
// directional light after the environment (as every NEE here).
template <typename T> V3<T> in_scattering(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w) {
    const V3<T> sun_dir = V3<T>::load(S.s.sun_dir), sun_L = V3<T>::load(S.s.sun_radiance);
    V3<T> ls_dir;
    V3<T> Ls_env = environment_sampler(S, rng, ls_dir);
    V3<T> Ls = transmittance(S, rng, x, ls_dir, nullptr) * Ls_env * phase(S, w, ls_dir);
    if (S.s.has_sun) Ls += transmittance(S, rng, x, sun_dir, nullptr) * sun_L * phase(S, w, sun_dir);
    V3<T> ws;
    T rho_s = phase_sampler(S, rng, w, ws);
    Counters dummy;
    Ls += rho_s * path_integrator_NEE(S, rng, x, ws, true, dummy);
    return S.albedo(x) * Ls;
}

// The scatter-gradient term at a transmittance-sampled position of the
// segment (x, w, d) (vr_path_integrator_NEE_DRTQ.h:156-165 and :249-259), on
// the segment's own stream (Rng::segment_stream).
template <typename T>
void drtq_scatter_term(const Scene<T>& S, Rng sec, V3<T> x, V3<T> w, T d, V3<T> W, V3<T> dL_dR) {
    T s_t, weight_t;
    sample_transmittance_position(S, sec, x, w, d, s_t, weight_t);
    V3<T> xs = x + w * s_t;
    V3<T> Ls = in_scattering(S, sec, xs, w);
    T sigma_t = S.sigma(xs);
    T mis_T = T(1) / (T(1) + sigma_t * sigma_t);
    S.sigma_bw(xs, mis_T * weight_t * dot(dL_dR, W * Ls));
}

// include/vr_path_integrator_NEE_DRTQ.h:58-260 path_integrator_NEE_DRTQ_bw:
// the DRT primal without a reservoir, and a scatter-gradient term on every
// segment of the replay.  Branch seed = Philox stream 1 for the light rays'
// adjoints (fork j of it beside fork j of the path's stream, as in DRT); each
// scatter term on its segment's stream.  A path stops at 2^24 - 1 segments.
template <typename T> void path_integrator_NEE_DRTQ_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, V3<T> dL_dR) {
    T tMin, tMax;
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    T d = tMax - tMin;
    if (d <= T(0)) return;
    Rng sec = rng;
    sec.stream = rng.stream + 1;
    sec.n = 0;
    sec.ntr = 0;
    (void)transmittance(S, rng, x, w, nullptr);
    transmittance_bw(S, sec, x, w, dot(dL_dR, S.environment(w)));
    V3<T> R(T(0)), W(T(1));
    const V3<T> ini_x = x, ini_w = w;
    const T ini_d = d;
    const T EPS = T(0.00000001);
    const V3<T> sun_dir = V3<T>::load(S.s.sun_dir), sun_L = V3<T>::load(S.s.sun_radiance);
    Rng before_path = rng;
    int bounces = 0;
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = ff.bk.query(S.s, x, w, md) * T(1.05) + T(0.1);
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        if ((T)rng.uniform() >= s / m) { d -= t; continue; }
        W *= S.albedo(x);
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        T T_nee = transmittance(S, rng, x, wnee, nullptr);
        R += W * T_nee * env * phase(S, w, wnee);
        if (S.s.has_sun) R += W * transmittance(S, rng, x, sun_dir, nullptr) * sun_L * phase(S, w, sun_dir);
        bool capped = S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces;
        V3<T> wo;
        W *= phase_sampler(S, rng, w, wo);
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
        if (all_less(W, EPS) || capped) break;
    }
    W = V3<T>(T(1));
    x = ini_x;
    w = ini_w;
    d = ini_d;
    rng = before_path;
    bounces = 0;
    uint32_t vertex = 0;  // scattering vertices so far: the next segment's number
    drtq_scatter_term(S, rng.segment_stream(0), x, w, d, W, dL_dR);
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = ff.bk.query(S.s, x, w, md) * T(1.05) + T(0.1);
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        T Pc = s / m;
        if ((T)rng.uniform() >= Pc) {
            S.sigma_bw(x, dot(dL_dR, -R / m / (T(1) - s / m)));
            d -= t;
            continue;
        }
        T dL_dsigma = dot(dL_dR, s * s / (T(1) + s * s) * R / s);
        W *= S.albedo(x);
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        T T_nee = transmittance(S, rng, x, wnee, nullptr);
        T ph_nee = phase(S, w, wnee);
        T T_sun = 0, ph_sun = 0;
        if (S.s.has_sun) {
            T_sun = transmittance(S, rng, x, sun_dir, nullptr);
            ph_sun = phase(S, w, sun_dir);
        }
        bool capped = S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces;
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        T dL_dTnee = dot(dL_dR, W * env * ph_nee);
        R -= W * T_nee * env * ph_nee;
        T dL_dTsun = 0;
        if (S.s.has_sun) {
            dL_dTsun = dot(dL_dR, W * sun_L * ph_sun);
            R -= W * T_sun * sun_L * ph_sun;
        }
        S.sigma_bw(x, dL_dsigma);
        transmittance_bw(S, sec, x, wnee, dL_dTnee);
        if (S.s.has_sun) transmittance_bw(S, sec, x, sun_dir, dL_dTsun);
        W *= rho;
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
        if (all_less(W, EPS) || capped || ++vertex + 1u >= (1u << 24)) break;
        drtq_scatter_term(S, rng.segment_stream(vertex), x, w, d, W, dL_dR);
    }
}

// include/vr_path_integrator_NEE_DRTDS.h:8-38 sample_collision_position_ds
// (majorant queried at the sample point, as in sample_transmittance_position).
template <typename T>
void sample_collision_position_ds(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T d, T epsilon, T& t, T& weight_t) {
    const T EPS = T(0.0000001);
    t = 0;
    weight_t = 1;
    for (int it = 0; it < (1 << 24); ++it) {
        T md;
        T m = vmax(EPS, S.majorant(x + w * t, w, md) + T(2) * epsilon + T(0.1));
        T dt = vmin(-std::log(T(1) - (T)rng.uniform()) / m, vmin(md, d - t));
        t += dt;
        if (dt >= md - EPS) continue;
        if (t >= d - EPS) break;
        T s = S.sigma(x + w * t);
        T Pc = (s + epsilon) / m;
        if ((T)rng.uniform() < Pc) {
            weight_t *= T(1) / (s + epsilon);
            return;
        }
        weight_t *= (T(1) - s / m) / (T(1) - Pc);
    }
    weight_t = 0;
}

// include/vr_path_integrator_NEE_DRTDS.h:40-253 path_integrator_NEE_DRTDS_bw:
// the DRT primal and reservoir; the replay scatters no MIS term at real
// collisions, and the reservoir term samples a defensive collision position.
template <typename T>
void path_integrator_NEE_DRTDS_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T epsilon, V3<T> dL_dR) {
    T tMin, tMax;
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    T d = tMax - tMin;
    if (d <= T(0)) return;
    Rng sec = rng;
    sec.stream = rng.stream + 1;
    sec.n = 0;
    sec.ntr = 0;
    (void)transmittance(S, rng, x, w, nullptr);
    transmittance_bw(S, sec, x, w, dot(dL_dR, S.environment(w)));
    V3<T> R(T(0)), W(T(1));
    V3<T> res_x = x, res_w = w, res_W = W;
    T res_P = 3, total_weight = 3;
    const V3<T> ini_x = x, ini_w = w;
    const T ini_d = d;
    const T EPS = T(0.00000001);
    const V3<T> sun_dir = V3<T>::load(S.s.sun_dir), sun_L = V3<T>::load(S.s.sun_radiance);
    Rng before_path = rng;
    int bounces = 0;
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = ff.bk.query(S.s, x, w, md) * T(1.05) + T(0.1);
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        if ((T)rng.uniform() >= s / m) { d -= t; continue; }
        W *= S.albedo(x);
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        T T_nee = transmittance(S, rng, x, wnee, nullptr);
        R += W * T_nee * env * phase(S, w, wnee);
        if (S.s.has_sun) R += W * transmittance(S, rng, x, sun_dir, nullptr) * sun_L * phase(S, w, sun_dir);
        bool capped = S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces;
        V3<T> wo;
        W *= phase_sampler(S, rng, w, wo);
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
        T current_P = W.x + W.y + W.z;
        total_weight += current_P;
        if ((T)rng.uniform() < current_P / total_weight) {
            res_P = current_P; res_W = W; res_x = x; res_w = w;
        }
        if (all_less(W, EPS) || capped) break;
    }
    W = V3<T>(T(1));
    x = ini_x;
    w = ini_w;
    d = ini_d;
    rng = before_path;
    bounces = 0;
    for (Flight<T> ff; d > EPS;) {
        T md;
        T m = ff.bk.query(S.s, x, w, md) * T(1.05) + T(0.1);
        T t = ff.sample(rng) / m;
        x += w * vmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(S.s); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        T s = S.sigma(x);
        if ((T)rng.uniform() >= s / m) {
            S.sigma_bw(x, dot(dL_dR, -R / m / (T(1) - s / m)));
            d -= t;
            continue;
        }
        V3<T> sa = S.albedo(x);
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        T T_nee = transmittance(S, rng, x, wnee, nullptr);
        T ph_nee = phase(S, w, wnee);
        T T_sun = 0, ph_sun = 0;
        if (S.s.has_sun) {
            T_sun = transmittance(S, rng, x, sun_dir, nullptr);
            ph_sun = phase(S, w, sun_dir);
        }
        bool capped = S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces;
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        W *= sa;
        T dL_dTnee = dot(dL_dR, W * env * ph_nee);
        R -= W * T_nee * env * ph_nee;
        T dL_dTsun = 0;
        if (S.s.has_sun) {
            dL_dTsun = dot(dL_dR, W * sun_L * ph_sun);
            R -= W * T_sun * sun_L * ph_sun;
        }
        transmittance_bw(S, sec, x, wnee, dL_dTnee);
        if (S.s.has_sun) transmittance_bw(S, sec, x, sun_dir, dL_dTsun);
        W *= rho;
        w = wo;
        S.boundary(x, w, tMin, d);
        ff.bk.reset();
        rng.advance();
        if (all_less(W, EPS) || capped) break;
    }
    S.boundary(res_x, res_w, tMin, d);
    T s_t, weight_t;
    sample_collision_position_ds(S, rng, res_x, res_w, d, epsilon, s_t, weight_t);
    if (weight_t > T(0)) {
        V3<T> xs = res_x + res_w * s_t;
        V3<T> ls_dir;
        V3<T> Ls_env = environment_sampler(S, rng, ls_dir);
        V3<T> Ls = transmittance(S, rng, xs, ls_dir, nullptr) * Ls_env * phase(S, res_w, ls_dir);
        if (S.s.has_sun) Ls += transmittance(S, rng, xs, sun_dir, nullptr) * sun_L * phase(S, res_w, sun_dir);
        V3<T> ws;
        T rho_s = phase_sampler(S, rng, res_w, ws);
        Counters dummy;
        Ls += rho_s * path_integrator_NEE(S, rng, xs, ws, true, dummy);
        Ls *= res_W * weight_t * S.albedo(xs);
        S.sigma_bw(xs, dot(dL_dR, Ls) * total_weight / res_P);
    }
}

// include/vr_path_integrator_NEE_SPS.h:1-59 sample_collision_position: delta
// tracking to a collision (majorant + 1e-6, queried at the current sample
// point: the reference queries it at the not yet written output point, which
// its constant majorant ignores), then, while MIS is allowed, a choice with
// MIS (beta 3) between that collision and a uniform point of the segment up to
// it; picking the uniform point makes it the path's singular vertex.
template <typename T>
bool sample_collision_position(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T d, V3<T>& xc, T& weight_xc,
                               T& sigma_xc, int& samples, bool& mis_allowed) {
    T t = 0;
    weight_xc = 0;
    sigma_xc = 0;
    samples = 0;
    xc = x;
    for (int it = 0; it < (1 << 24); ++it) {
        T md;
        T m = S.majorant(xc, w, md) + T(0.000001);
        T dt = vmin(-std::log(T(1) - (T)rng.uniform()) / m, vmin(md, d - t));
        t += dt;
        xc = w * t + x;
        if (dt >= md - T(0.0000001)) continue;
        if (t >= d - T(0.0000001)) break;
        T s = S.sigma(xc);
        samples++;
        if ((T)rng.uniform() < s / m) {
            weight_xc = 1;
            sigma_xc = s;
            break;
        }
    }
    if (!mis_allowed) return false;
    T powered_c = sigma_xc * sigma_xc * sigma_xc;  // pow(sigma, MIS_BETA) with MIS_BETA = 3
    T mis_wc = weight_xc * powered_c / (T(1) + powered_c);
    T u = (T)rng.uniform();
    V3<T> xf = xc * (T(1) - u) + x * u;
    T sigma_f = S.sigma(xf);
    T powered_f = sigma_f * sigma_f * sigma_f;
    T mis_wf = t / (T(1) + powered_f);
    weight_xc = mis_wc + mis_wf;
    if ((T)rng.uniform() * weight_xc < mis_wf) {
        xc = xf;
        sigma_xc = sigma_f;
        mis_allowed = false;
        return true;
    }
    return false;
}

// include/vr_path_integrator_NEE_SPS.h:88-101 st_tau_bw (stratified bins)
template <typename T> void st_tau_bw(const Scene<T>& S, Rng& rng, V3<T> a, V3<T> b, int bins, T dL_dtau) {
    if (dL_dtau == T(0) || bins == 0) return;
    T d = std::sqrt(dot(a - b, a - b));
    T g = dL_dtau * d / T(bins);
    for (int i = 0; i < bins; ++i) {
        T f = (T(i) + (T)rng.uniform()) / T(bins);
        S.sigma_bw(b * (T(1) - f) + a * f, g);
    }
}

// include/vr_path_integrator_NEE_SPS.h:104-263 path_integrator_NEE_SPS_bw
// (emission ignored, as in the reference; directional light and bounce cap as
// in the other adjoints).
template <typename T> void path_integrator_NEE_SPS_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, V3<T> dL_dR) {
    T tMin, tMax;
    S.boundary(x, w, tMin, tMax);
    x += w * tMin;
    T d = tMax - tMin;
    if (d <= T(0)) return;
    Rng sec = rng;
    sec.stream = rng.stream + 1;
    sec.n = 0;
    sec.ntr = 0;
    (void)transmittance(S, rng, x, w, nullptr);
    transmittance_bw(S, sec, x, w, dot(dL_dR, S.environment(w)));
    const V3<T> sun_dir = V3<T>::load(S.s.sun_dir), sun_L = V3<T>::load(S.s.sun_radiance);
    V3<T> R(T(0)), Rf(T(0)), W(T(1));
    T W_singular = 1;
    bool mis_allowed = true;
    const V3<T> ini_x = x, ini_w = w;
    const T ini_d = d;
    const T EPS = T(0.00001);
    Rng before_path = rng;
    int bounces = 0;
    for (int it = 0; it < (1 << 24); ++it) {
        T weight_xc, sigma_xc;
        V3<T> xc;
        int samples;
        if (sample_collision_position(S, rng, x, w, d, xc, weight_xc, sigma_xc, samples, mis_allowed))
            W_singular = sigma_xc;
        if (weight_xc == T(0)) break;
        x = xc;
        W *= weight_xc * S.albedo(x);
        V3<T> wnee;
        V3<T> nee_env = environment_sampler(S, rng, wnee);
        T nee_T = transmittance(S, rng, x, wnee, nullptr);
        V3<T> added_R = W * nee_T * phase(S, w, wnee) * nee_env;
        if (S.s.has_sun) added_R += W * transmittance(S, rng, x, sun_dir, nullptr) * phase(S, w, sun_dir) * sun_L;
        if (mis_allowed) R += added_R;
        else Rf += added_R;
        bool capped = S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces;
        V3<T> wo;
        W *= phase_sampler(S, rng, w, wo);
        w = wo;
        S.boundary(x, w, tMin, d);
        if (all_less(W, EPS) || capped) break;
    }
    W = V3<T>(T(1));
    mis_allowed = true;
    x = ini_x;
    w = ini_w;
    d = ini_d;
    V3<T> prev_x = x;
    rng = before_path;
    bounces = 0;
    for (int it = 0; it < (1 << 24); ++it) {
        T weight_xc, sigma_xc;
        V3<T> xc;
        int samples;
        bool singular = sample_collision_position(S, rng, x, w, d, xc, weight_xc, sigma_xc, samples, mis_allowed);
        if (weight_xc == T(0)) break;
        V3<T> further_R = R + W_singular * Rf;
        T k = dot(dL_dR, further_R);
        T dL_dtau = -k;
        T dL_dsigma = singular ? dot(dL_dR, Rf) : k / vmax(T(0.001), sigma_xc);
        x = xc;
        W *= weight_xc;
        W *= S.albedo(x);
        V3<T> wnee;
        V3<T> env = environment_sampler(S, rng, wnee);
        T T_nee = transmittance(S, rng, x, wnee, nullptr);
        T ph_nee = phase(S, w, wnee);
        T T_sun = 0, ph_sun = 0;
        if (S.s.has_sun) {
            T_sun = transmittance(S, rng, x, sun_dir, nullptr);
            ph_sun = phase(S, w, sun_dir);
        }
        bool capped = S.s.max_bounces > 0 && ++bounces >= S.s.max_bounces;
        V3<T> wo;
        T rho = phase_sampler(S, rng, w, wo);
        const T fs = mis_allowed ? T(1) : W_singular;
        T dL_dTnee = dot(dL_dR, W * fs * env * ph_nee);
        V3<T> added_R = W * T_nee * ph_nee * env;
        T dL_dTsun = 0;
        if (S.s.has_sun) {
            dL_dTsun = dot(dL_dR, W * fs * sun_L * ph_sun);
            added_R += W * T_sun * ph_sun * sun_L;
        }
        if (mis_allowed) R -= added_R;
        else Rf -= added_R;
        S.sigma_bw(x, dL_dsigma);
        st_tau_bw(S, sec, x, prev_x, samples > 1 ? samples : 1, dL_dtau);
        transmittance_bw(S, sec, x, wnee, dL_dTnee);
        if (S.s.has_sun) transmittance_bw(S, sec, x, sun_dir, dL_dTsun);
        W *= rho;
        w = wo;
        S.boundary(x, w, tMin, d);
        if (all_less(W, EPS) || capped) break;
        prev_x = x;
    }
}

// include/maps/sensor_perspective_camera.h:1-27
template <typename T>
void camera_ray(const orc_camera& cam, int view, int row, int col, Rng& rng, V3<T>& x, V3<T>& w) {
    const float* p = cam.poses + 9 * (int64_t)view;
    V3<T> o = V3<T>::load(p), dd = V3<T>::load(p + 3), n = V3<T>::load(p + 6);
    T sx_ = T(0.5), sy_ = T(0.5);
    if (cam.jittered) { sx_ = (T)rng.uniform(); sy_ = (T)rng.uniform(); }
    T znear = (T)cam.znear;
    T sx = ((T(col) + sx_) * T(2) - T(cam.width)) * znear / T(cam.height);
    T sy = ((T(row) + sy_) * T(2) - T(cam.height)) * znear / T(cam.height);
    T sz = znear / std::tan((T)cam.fov * T(0.5));
    V3<T> zaxis = normalize(dd);
    V3<T> xaxis = normalize(cross(n, zaxis));
    V3<T> yaxis = cross(zaxis, xaxis);
    w = xaxis * sx + yaxis * sy + zaxis * sz;
    x = o + w;
    w = normalize(w);
}

inline uint64_t capture_path_id(int64_t pixel, int s, int64_t npix) { return (uint64_t)s * (uint64_t)npix + (uint64_t)pixel; }

// Sensors of a capture (SensorsBase.capture, _maps.py:1741-1749, and the
// capture kernel's index decoding, _maps.py:560-577): every pixel of every
// view in raster order, or the (view, row, col) triples of a sensors batch.
inline int64_t camera_npix(const orc_camera& cam) {
    return cam.sensors ? cam.n_sensors : (int64_t)cam.views * cam.height * cam.width;
}
inline void camera_pixel(const orc_camera& cam, int64_t p, int& view, int& row, int& col) {
    if (cam.sensors) {
        view = (int)cam.sensors[3 * p]; row = (int)cam.sensors[3 * p + 1]; col = (int)cam.sensors[3 * p + 2];
        return;
    }
    view = (int)(p / ((int64_t)cam.height * cam.width));
    int rem = (int)(p % ((int64_t)cam.height * cam.width));
    row = rem / cam.width;
    col = rem % cam.width;
}

// pixel of a radiance-cache training path: the path's first draw, scaled to npix
inline int64_t random_pixel(Rng& rng, int64_t npix) { return (int64_t)(((uint64_t)rng.u32() * (uint64_t)npix) >> 32); }

// ---------------------------------------------------------------------------
// Collision sampling and collision integrators (_maps.py:2714-2852).
// ---------------------------------------------------------------------------
// include/vr_collision_sampler_DT.h:6-43: a delta-tracking collision along the
// ray; returns C (1 at a collision, else 0), the collision distance out_t from
// x and out_T (0 at a collision, else 1).  The free flight carries its residual
// optical depth across majorant-brick faces, as every tracker here does.
template <typename T>
T collision_sampler_DT(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T& out_t, T& out_T, int64_t* steps) {
    out_T = T(1);
    out_t = T(0);
    T C = T(0);
    T tMin, tMax;
    if (!S.boundary(x, w, tMin, tMax)) return C;
    const T d = tMax - tMin;
    x += w * tMin;
    T t = T(0);
    Flight<T> ff;
    for (; ff.it < (1 << 24); ++ff.it) {
        T md;
        const T maj = ff.bk.query(S.s, x, w, md);
        const T tau = ff.sample(rng);
        if (steps) ++*steps;
        const bool crosses = tau > md * maj;
        T dt = crosses ? md : tau / maj;
        dt = vmin(dt, d);
        x += w * dt;
        t += dt;
        if (t >= d - T(0.0000001)) break;
        if (crosses) { ff.cross(maj, md); ff.bk.advance(S.s); continue; }
        ff.used();
        ff.bk.move(dt);
        if ((T)rng.uniform() < S.sigma(x) / maj) {
            out_T = T(0);
            C = T(1);
            break;
        }
    }
    out_t = tMin + t;
    return C;
}

// include/vr_collision_sampler_DT.h:45-134: the defensively sampled walk
// (majorant + 2 eps, Pc = (sigma + eps) / majorant) for the estimate, then the
// same draws again scattering dL/dsigma at its collisions.
template <typename T>
void collision_sampler_DT_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, T eps, T dL_dC, T dL_dT) {
    T tMin, tMax;
    if (!S.boundary(x, w, tMin, tMax)) return;
    const Rng before = rng;
    T out_T = T(1), C = T(0), s_t = T(0);
    const T d = tMax - tMin;
    x += w * tMin;
    const V3<T> ini_x = x;
    for (int pass = 0; pass < 2; ++pass) {
        T t = T(0);
        Flight<T> ff;
        for (; ff.it < (1 << 24); ++ff.it) {
            T md;
            const T maj = vmax(T(0.0000000001), ff.bk.query(S.s, x, w, md) + T(2) * eps);
            const T tau = ff.sample(rng);
            const bool crosses = tau > md * maj;
            T dt = crosses ? md : tau / maj;
            dt = vmin(dt, d);
            x += w * dt;
            t += dt;
            if (t >= d - T(0.0000001)) break;
            if (crosses) { ff.cross(maj, md); ff.bk.advance(S.s); continue; }
            ff.used();
            ff.bk.move(dt);
            const T s = S.sigma(x);
            const T Pc = (s + eps) / maj;
            const bool hit = (T)rng.uniform() < Pc;
            if (pass == 0) {
                if (hit) {
                    out_T = T(0);
                    C = T(1);
                    s_t = s / maj / Pc;
                    break;
                }
                out_T *= (T(1) - s / maj) / (T(1) - Pc);
            } else if (hit) {
                S.sigma_bw(x, dL_dC * (C / Pc) * (T(1) / maj));
                break;
            } else {
                const T g = (dL_dT * out_T + dL_dC * C * s_t) / ((T(1) - s / maj) / (T(1) - Pc)) / (T(1) - Pc);
                S.sigma_bw(x, g * (T(-1) / maj));
            }
        }
        rng = before;
        x = ini_x;
    }
}

// Exitance radiance R(x, w_out) of a collision integrator (w_out = -ray
// direction), by the medium's exitance_mode:
//   0  the emission map (const or Grid3D): ds.exitance_radiance = ds.emission
//   1  MCScatteredRadiance (include/maps/scattered_radiance_mc.h):
//      sa(x) * rho * radiance(x, wo), (rho, wo) = phase_sampler(x, -w_out)
//   2  MCScatteredEmittedRadiance (include/maps/scattered_emitted_radiance_mc.h):
//      the same plus (1 - sa) * emission(x)
// where radiance(x, wo) = transmittance(x, wo) * environment (the
// ds.transmittance * ds.environment.after(ray_direction) of _objects.py:270).
// rng is the evaluation's own stream; the transmittance forks from it.
template <typename T> V3<T> exitance(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> wout) {
    const int mode = S.s.exitance_mode;
    if (mode == 0) return S.emission_at(x);
    V3<T> wo;
    const T rho = phase_sampler(S, rng, -wout, wo);
    const V3<T> sa = S.albedo(x);
    const V3<T> rad = S.environment(wo) * transmittance(S, rng, x, wo, (int64_t*)nullptr);
    V3<T> R = sa * rho * rad;
    if (mode == 2) R += (V3<T>(T(1)) - sa) * S.emission_at(x);
    return R;
}
// Adjoint of exitance() on the same draws.  The reference's backward of the
// scattered maps hands (w, dL/dR) to the radiance map and drops the dL/dR
// factor of the emission term of dL/dsa; here each factor gets the adjoint of
// the forward's own expression.
template <typename T> void exitance_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> wout, V3<T> dL) {
    const int mode = S.s.exitance_mode;
    if (mode == 0) { S.emission_bw(x, dL); return; }
    V3<T> wo;
    const T rho = phase_sampler(S, rng, -wout, wo);
    const V3<T> sa = S.albedo(x);
    Rng tr_rng = rng;
    const T Tr = transmittance(S, rng, x, wo, (int64_t*)nullptr);
    const V3<T> env = S.environment(wo);
    const V3<T> rad = env * Tr;
    V3<T> dL_dsa = dL * rad * rho;
    const V3<T> dL_drad = dL * sa * rho;
    if (mode == 2) {
        const V3<T> em = S.emission_at(x);
        dL_dsa -= dL * em;
        S.emission_bw(x, dL * (V3<T>(T(1)) - sa));
    }
    S.albedo_bw(x, dL_dsa);
    transmittance_bw(S, tr_rng, x, wo, dot(dL_drad, env));
}

// Streams of one collision-integrator path: the collision sampler on stream 2,
// its adjoint on stream 4, exitance evaluation k on stream (k + 1) << 16 (its
// transmittance on the fork after it).
inline uint32_t exitance_stream(int64_t k) { return (uint32_t)((k + 1) & 0x7fff) << 16; }

// include/maps/collision_integrator_mc.h:8-18 (MCCollisionIntegrator FORWARD)
template <typename T> V3<T> collision_integrator_MC(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, Counters& c) {
    Rng cs = rng.with_stream(2);
    T t, Tt;
    const T C = collision_sampler_DT(S, cs, x, w, t, Tt, &c.steps);
    if (C != T(0)) ++c.vertices;
    const V3<T> xt = w * t + x;
    Rng xr = rng.with_stream(exitance_stream(0));
    const V3<T> eR = C != T(0) ? exitance(S, xr, xt, -w) : V3<T>(T(0));
    return eR * C + S.environment(w) * Tt;
}
// include/maps/collision_integrator_mc.h:20-41 (BACKWARD): the forward's
// collision (same stream), the sampler's adjoint on its own stream, the
// exitance's adjoint on the forward's exitance draws.
template <typename T> void collision_integrator_MC_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, V3<T> dL) {
    Rng cs = rng.with_stream(2);
    T t, Tt;
    const T C = collision_sampler_DT(S, cs, x, w, t, Tt, (int64_t*)nullptr);
    const V3<T> xt = w * t + x;
    Rng xr = rng.with_stream(exitance_stream(0));
    const V3<T> eR = C != T(0) ? exitance(S, xr, xt, -w) : V3<T>(T(0));
    const V3<T> env = S.environment(w);
    Rng cb = rng.with_stream(4);
    collision_sampler_DT_bw(S, cb, x, w, (T)S.s.ds_epsilon, dot(dL, eR), dot(dL, env));
    if (C != T(0)) {
        Rng xb = rng.with_stream(exitance_stream(0));
        exitance_bw(S, xb, xt, -w, dL * C);
    }
}

// include/vr_collision_integrator_DDA.h:1-82: the DDA walk of the grid with
// one random point per cell (the path stream): per cell the homogeneous
// transmittance exp(-dt sigma(point)) and the exitance at the point.
template <typename T> V3<T> collision_integrator_DDA(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, Counters& c) {
    const V3<T> env = S.environment(w);
    DDA<T> dda(S, x, w);
    if (!dda.valid) return env;
    T Tr = T(1), ct = T(0);
    V3<T> R(T(0));
    T s[2][2][2];
    int64_t k = 0;
    while (ct < dda.d - T(0.0001)) {
        const T nt = vmin(dda.d, vmin(dda.alpha.x, vmin(dda.alpha.y, dda.alpha.z)));
        dda.load_cell(s);
        const T cell_t = mix(ct, nt, (T)rng.uniform());
        const T sv = interpolated_sigma(dda.ialpha(cell_t), s);
        const T vt = std::exp(-(nt - ct) * sv);
        Rng xr = rng.with_stream(exitance_stream(k));
        const V3<T> Le = exitance(S, xr, dda.x + w * cell_t, -w);
        R += Le * (Tr * (T(1) - vt));
        Tr *= vt;
        ++c.steps;
        ct = nt;
        dda.step();
        ++k;
    }
    return R + env * Tr;
}
// include/vr_collision_integrator_DDA.h:85-207: the same walk for fw_T and the
// emitted part, then a replay from the same cell draws scattering
// dL/dsigma = dL/dR . (T Le - fw_T env - R_rest) dt and the exitance adjoint.
template <typename T> void collision_integrator_DDA_bw(const Scene<T>& S, Rng& rng, V3<T> x, V3<T> w, V3<T> dL) {
    if (dL.x == T(0) && dL.y == T(0) && dL.z == T(0)) return;
    DDA<T> dda(S, x, w);
    if (!dda.valid) return;
    const Rng before = rng;
    T Tr = T(1), ct = T(0);
    V3<T> R(T(0));
    T s[2][2][2];
    int64_t k = 0;
    while (ct < dda.d - T(0.0001)) {
        const T nt = vmin(dda.d, vmin(dda.alpha.x, vmin(dda.alpha.y, dda.alpha.z)));
        dda.load_cell(s);
        const T cell_t = mix(ct, nt, (T)rng.uniform());
        const T sv = interpolated_sigma(dda.ialpha(cell_t), s);
        const T vt = std::exp(-(nt - ct) * sv);
        Rng xr = rng.with_stream(exitance_stream(k));
        R += exitance(S, xr, dda.x + w * cell_t, -w) * (Tr * (T(1) - vt));
        Tr *= vt;
        ct = nt;
        dda.step();
        ++k;
    }
    const V3<T> env = S.environment(w);
    const T fw_T = Tr;
    rng = before;
    dda.reset_march();
    Tr = T(1);
    ct = T(0);
    k = 0;
    T g[2][2][2];
    while (ct < dda.d - T(0.0001)) {
        const T nt = vmin(dda.d, vmin(dda.alpha.x, vmin(dda.alpha.y, dda.alpha.z)));
        dda.load_cell(s);
        const T cell_t = mix(ct, nt, (T)rng.uniform());
        const V3<T> a = dda.ialpha(cell_t);
        const T sv = interpolated_sigma(a, s);
        const T dt = nt - ct;
        const T vt = std::exp(-dt * sv);
        const V3<T> xp = dda.x + w * cell_t;
        Rng xr = rng.with_stream(exitance_stream(k));
        const V3<T> Le = exitance(S, xr, xp, -w);
        Rng xb = rng.with_stream(exitance_stream(k));
        exitance_bw(S, xb, xp, -w, dL * (Tr * (T(1) - vt)));
        R -= Le * (Tr * (T(1) - vt));
        Tr *= vt;
        const T dL_dsigma = dot(dL, (Le * Tr - env * fw_T - R) * dt);
        interpolated_sigma_bw(a, dL_dsigma, g);
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx)
                    S.sigma_at_bw(dda.cell[0] + dx, dda.cell[1] + dy, dda.cell[2] + dz, g[dz][dy][dx]);
        ct = nt;
        dda.step();
        ++k;
    }
}

// integrator: 0 NEE, 1 DT, 2 MC collision integrator, 3 DDA collision integrator
template <typename T> V3<T> radiance(const Scene<T>& S, int integrator, Rng& rng, V3<T> x, V3<T> w, Counters& c) {
    if (integrator == 2) return collision_integrator_MC(S, rng, x, w, c);
    if (integrator == 3) return collision_integrator_DDA(S, rng, x, w, c);
    return integrator == 0 ? path_integrator_NEE(S, rng, x, w, false, c) : path_integrator_DT(S, rng, x, w, c);
}
template <typename T> void radiance_bw(const Scene<T>& S, int bw_mode, Rng& rng, V3<T> x, V3<T> w, V3<T> dL) {
    if (bw_mode == 0) path_integrator_NEE_DS_bw(S, rng, x, w, (T)S.s.ds_epsilon, dL);
    else if (bw_mode == 1) path_integrator_DT_bw(S, rng, x, w, (T)S.s.ds_epsilon, dL);
    else if (bw_mode == 2) path_integrator_NEE_DRT_bw(S, rng, x, w, dL);
    else if (bw_mode == 3) path_integrator_NEE_DRTQ_bw(S, rng, x, w, dL);
    else if (bw_mode == 4) path_integrator_NEE_DRTDS_bw(S, rng, x, w, (T)S.s.ds_epsilon, dL);
    else if (bw_mode == 5) path_integrator_NEE_SPS_bw(S, rng, x, w, dL);
    else if (bw_mode == 6) collision_integrator_MC_bw(S, rng, x, w, dL);
    else collision_integrator_DDA_bw(S, rng, x, w, dL);
}

template <typename T> void transmittance_fw_impl(const orc_scene* s, int32_t mode, const float* rays, int64_t n, uint64_t seed, float* Tout) {
    orc_scene sc = *s;
    sc.transmittance_mode = mode;
    Scene<T> S(sc);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        Rng rng(seed, (uint64_t)i, 0);
        Tout[i] = (float)transmittance(S, rng, V3<T>::load(rays + 6 * i), V3<T>::load(rays + 6 * i + 3), (int64_t*)nullptr);
    }
}
}  // namespace

// ===========================================================================
extern "C" {

void orc_set_threads(int32_t n) { omp_set_num_threads(n > 0 ? n : 1); }
int32_t orc_get_threads(void) { return omp_get_max_threads(); }

void orc_philox4x32_10(uint32_t key0, uint32_t key1, const uint32_t ctr[4], uint32_t out[4]) { philox(key0, key1, ctr, out); }

void orc_random_sequence(uint64_t seed, uint64_t path, uint32_t stream, uint32_t start, int32_t n, float* out) {
    Rng r(seed, path, stream);
    r.n = start;
    for (int i = 0; i < n; ++i) out[i] = r.uniform();
}

void orc_ray_box(const float* rays, int64_t n, const float bmin[3], const float bmax[3], float* out2) {
    for (int64_t i = 0; i < n; ++i) {
        float a, b;
        ray_box_intersection(V3<float>::load(rays + 6 * i), V3<float>::load(rays + 6 * i + 3), V3<float>::load(bmin),
                             V3<float>::load(bmax), a, b);
        out2[2 * i] = a;
        out2[2 * i + 1] = b;
    }
}

void orc_grid3d_fw(const orc_grid* g, const float bmin[3], const float inv_bsize[3], const float* x, int64_t n, float* out) {
    orc_scene sc;
    std::memset(&sc, 0, sizeof(sc));
    std::memcpy(sc.bmin, bmin, 12);
    std::memcpy(sc.inv_bsize, inv_bsize, 12);
    Scene<float> S(sc);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) S.grid_fw(*g, V3<float>::load(x + 3 * i), out + (int64_t)g->C * i);
}

void orc_grid3d_bw(const orc_grid* g, const float bmin[3], const float inv_bsize[3], const float* x, const float* dout, int64_t n) {
    orc_scene sc;
    std::memset(&sc, 0, sizeof(sc));
    std::memcpy(sc.bmin, bmin, 12);
    std::memcpy(sc.inv_bsize, inv_bsize, 12);
    Scene<float> S(sc);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) S.grid_bw(*g, V3<float>::load(x + 3 * i), dout + (int64_t)g->C * i);
}

// Majorant grid (extension): brick b covers cells [b*B, (b+1)*B); its bound is
// the max over nodes [b*B-1, (b+1)*B+1] clamped to the grid (the trilinear
// stencil of every point in the brick plus a one-node apron).
void orc_majorant_build(const orc_grid* g, int32_t brick, float* out, int32_t dims_out[3]) {
    int dim[3] = {g->W - 1, g->H - 1, g->D - 1};
    int M[3];
    for (int i = 0; i < 3; ++i) M[i] = (dim[i] + brick - 1) / brick;
    if (dims_out) { dims_out[0] = M[0]; dims_out[1] = M[1]; dims_out[2] = M[2]; }
    if (!out) return;
#pragma omp parallel for collapse(2) schedule(static)
    for (int mz = 0; mz < M[2]; ++mz)
        for (int my = 0; my < M[1]; ++my)
            for (int mx = 0; mx < M[0]; ++mx) {
                float m = 0.0f;
                int lo[3] = {mx * brick - 1, my * brick - 1, mz * brick - 1};
                int hi[3] = {(mx + 1) * brick + 1, (my + 1) * brick + 1, (mz + 1) * brick + 1};
                for (int i = 0; i < 3; ++i) { lo[i] = std::max(lo[i], 0); hi[i] = std::min(hi[i], dim[i]); }
                for (int z = lo[2]; z <= hi[2]; ++z)
                    for (int y = lo[1]; y <= hi[1]; ++y)
                        for (int x = lo[0]; x <= hi[0]; ++x)
                            m = std::max(m, g->data[(((int64_t)z * g->H + y) * g->W + x) * g->C]);
                out[((int64_t)mz * M[1] + my) * M[0] + mx] = m;
            }
}

void orc_majorant_query(const orc_scene* s, const float* rays, int64_t n, float* out2) {
    Scene<float> S(*s);
    for (int64_t i = 0; i < n; ++i) {
        float md;
        out2[2 * i] = S.majorant(V3<float>::load(rays + 6 * i), V3<float>::load(rays + 6 * i + 3), md);
        out2[2 * i + 1] = md;
    }
}

void orc_transmittance_fw(const orc_scene* s, int32_t mode, const float* rays, int64_t n, uint64_t seed, int32_t fp64, float* T) {
    if (fp64) transmittance_fw_impl<double>(s, mode, rays, n, seed, T);
    else transmittance_fw_impl<float>(s, mode, rays, n, seed, T);
}
void orc_transmittance_bw(const orc_scene* s, int32_t mode, const float* rays, int64_t n, uint64_t seed, const float* dL_dT) {
    orc_scene sc = *s;
    sc.transmittance_mode = mode;
    Scene<float> S(sc);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        Rng rng(seed, (uint64_t)i, 0);
        transmittance_bw(S, rng, V3<float>::load(rays + 6 * i), V3<float>::load(rays + 6 * i + 3), dL_dT[i]);
    }
}

// The DDA's optical depth in FP64 (vr_transmittance_DDA.h:1-59 without the
// final exp): the quantity whose central differences check the DDA adjoint.
void orc_dda_tau_fp64(const orc_scene* s, int32_t exact, const float* rays, int64_t n, double* tau) {
    Scene<double> S(*s);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        DDA<double> dda(S, V3<double>::load(rays + 6 * i), V3<double>::load(rays + 6 * i + 3));
        tau[i] = dda.valid ? dda.tau(exact != 0, nullptr) : 0.0;
    }
}

// FP64 fine ray-march (extension, reference for the DDA modes): tau over the
// same clipped segment, split into `substeps` pieces per cell size along the
// ray, each integrated with two-point Gauss-Legendre of the trilinear field
// read through vr_sigma_grid.h's clamping lookup.
void orc_tau_raymarch_fp64(const orc_scene* s, const float* rays, int64_t n, int32_t substeps, double* tau) {
    Scene<double> S(*s);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        V3<double> x = V3<double>::load(rays + 6 * i), w = V3<double>::load(rays + 6 * i + 3);
        DDA<double> dda(S, x, w);
        if (!dda.valid) { tau[i] = 0.0; continue; }
        const int dim[3] = {s->sigma.W - 1, s->sigma.H - 1, s->sigma.D - 1};
        V3<double> fdim(dim[0], dim[1], dim[2]);
        double cell = std::min(dda.cell_size.x, std::min(dda.cell_size.y, dda.cell_size.z));
        double h = cell / substeps;
        int64_t nsteps = (int64_t)std::ceil(dda.d / h);
        if (nsteps < 1) nsteps = 1;
        h = dda.d / (double)nsteps;
        auto field = [&](double t) {
            V3<double> p = (dda.x + dda.w * t - dda.bmin) * fdim / dda.box_size;
            int c[3];
            double a[3];
            for (int k = 0; k < 3; ++k) {
                double f = std::floor(p[k]);
                c[k] = std::min(std::max((int)f, 0), dim[k] - 1);
                a[k] = p[k] - c[k];
            }
            double sg[2][2][2];
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx) sg[dz][dy][dx] = S.sigma_at(c[0] + dx, c[1] + dy, c[2] + dz);
            return interpolated_sigma(V3<double>(a[0], a[1], a[2]), sg);
        };
        double acc = 0.0;
        for (int64_t k = 0; k < nsteps; ++k) {
            double mid = (k + 0.5) * h, off = h * DDA<double>::GL;
            acc += 0.5 * h * (field(mid - off) + field(mid + off));
        }
        tau[i] = acc;
    }
}

void orc_phase_sample(const orc_scene* s, const float* w_in, int64_t n, uint64_t seed, float* out4) {
    Scene<float> S(*s);
    for (int64_t i = 0; i < n; ++i) {
        Rng rng(seed, (uint64_t)i, 0);
        V3<float> wo;
        float rho = phase_sampler(S, rng, V3<float>::load(w_in + 3 * i), wo);
        out4[4 * i] = rho; out4[4 * i + 1] = wo.x; out4[4 * i + 2] = wo.y; out4[4 * i + 3] = wo.z;
    }
}

void orc_env_sample(const orc_scene* s, int64_t n, uint64_t seed, float* out6) {
    Scene<float> S(*s);
    for (int64_t i = 0; i < n; ++i) {
        Rng rng(seed, (uint64_t)i, 0);
        V3<float> wo;
        V3<float> e = environment_sampler(S, rng, wo);
        out6[6 * i] = e.x; out6[6 * i + 1] = e.y; out6[6 * i + 2] = e.z;
        out6[6 * i + 3] = wo.x; out6[6 * i + 4] = wo.y; out6[6 * i + 5] = wo.z;
    }
}

void orc_camera_rays(const orc_camera* cam, int32_t spp, uint64_t seed, float* out6) {
    int64_t npix = camera_npix(*cam);
    for (int s = 0; s < spp; ++s)
        for (int64_t p = 0; p < npix; ++p) {
            int view, row, col;
            camera_pixel(*cam, p, view, row, col);
            Rng rng(seed, capture_path_id(p, s, npix), 0);
            V3<float> x, w;
            camera_ray(*cam, view, row, col, rng, x, w);
            float* o = out6 + 6 * ((int64_t)s * npix + p);
            o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = w.x; o[4] = w.y; o[5] = w.z;
        }
}

void orc_radiance_fw(const orc_scene* s, int32_t integrator, const float* rays, int64_t n, uint64_t seed, float* R, orc_counters* c) {
    Scene<float> S(*s);
    int64_t verts = 0, steps = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : verts, steps)
    for (int64_t i = 0; i < n; ++i) {
        Rng rng(seed, (uint64_t)i, 0);
        Counters cnt;
        V3<float> r = radiance(S, integrator, rng, V3<float>::load(rays + 6 * i), V3<float>::load(rays + 6 * i + 3), cnt);
        R[3 * i] = r.x; R[3 * i + 1] = r.y; R[3 * i + 2] = r.z;
        verts += cnt.vertices;
        steps += cnt.steps;
    }
    if (c) { c->paths = n; c->vertices = verts; c->steps = steps; }
}

// DeltatrackingCollisionSampler as a map (include/maps/collision_sampler_dt.h):
// ray i draws from stream 2 of path i (its adjoint from stream 4), as inside
// the MC collision integrator.
void orc_collision_sample_fw(const orc_scene* s, const float* rays, int64_t n, uint64_t seed, float* out3) {
    Scene<float> S(*s);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        Rng rng(seed, (uint64_t)i, 2);
        float t, Tt;
        const float C = collision_sampler_DT(S, rng, V3<float>::load(rays + 6 * i), V3<float>::load(rays + 6 * i + 3), t,
                                             Tt, (int64_t*)nullptr);
        out3[3 * i] = C;
        out3[3 * i + 1] = t;
        out3[3 * i + 2] = Tt;
    }
}
void orc_collision_sample_bw(const orc_scene* s, const float* rays, int64_t n, uint64_t seed, const float* dL_dout3) {
    Scene<float> S(*s);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        Rng rng(seed, (uint64_t)i, 4);
        collision_sampler_DT_bw(S, rng, V3<float>::load(rays + 6 * i), V3<float>::load(rays + 6 * i + 3),
                                (float)s->ds_epsilon, dL_dout3[3 * i], dL_dout3[3 * i + 2]);
    }
}

void orc_radiance_bw(const orc_scene* s, int32_t bw_mode, const float* rays, int64_t n, uint64_t seed, const float* dL_dR) {
    Scene<float> S(*s);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        Rng rng(seed, (uint64_t)i, 0);
        radiance_bw(S, bw_mode, rng, V3<float>::load(rays + 6 * i), V3<float>::load(rays + 6 * i + 3),
                    V3<float>::load(dL_dR + 3 * i));
    }
}

void orc_capture_fw(const orc_scene* s, int32_t integrator, const orc_camera* cam, int32_t spp, uint64_t seed, float* rgb, orc_counters* c) {
    Scene<float> S(*s);
    int64_t npix = camera_npix(*cam);
    int64_t verts = 0, steps = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : verts, steps)
    for (int64_t p = 0; p < npix; ++p) {
        int view, row, col;
        camera_pixel(*cam, p, view, row, col);
        V3<float> acc(0.0f);
        Counters cnt;
        for (int sidx = 0; sidx < spp; ++sidx) {
            Rng rng(seed, capture_path_id(p, sidx, npix), 0);
            V3<float> x, w;
            camera_ray(*cam, view, row, col, rng, x, w);
            acc += radiance(S, integrator, rng, x, w, cnt);
        }
        rgb[3 * p] = acc.x / (float)spp;
        rgb[3 * p + 1] = acc.y / (float)spp;
        rgb[3 * p + 2] = acc.z / (float)spp;
        verts += cnt.vertices;
        steps += cnt.steps;
    }
    if (c) { c->paths = npix * spp; c->vertices = verts; c->steps = steps; }
}

void orc_capture_fw_fp64(const orc_scene* s, const orc_camera* cam, int32_t spp, uint64_t seed, double* rgb) {
    Scene<double> S(*s);
    int64_t npix = camera_npix(*cam);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t p = 0; p < npix; ++p) {
        int view, row, col;
        camera_pixel(*cam, p, view, row, col);
        V3<double> acc(0.0);
        Counters cnt;
        for (int sidx = 0; sidx < spp; ++sidx) {
            Rng rng(seed, capture_path_id(p, sidx, npix), 0);
            V3<double> x, w;
            camera_ray(*cam, view, row, col, rng, x, w);
            acc += path_integrator_NEE(S, rng, x, w, false, cnt) * (1.0 / (double)spp);
        }
        rgb[3 * p] = acc.x;
        rgb[3 * p + 1] = acc.y;
        rgb[3 * p + 2] = acc.z;
    }
}

void orc_capture_prefix(const orc_scene* s, const orc_camera* cam, int32_t spp, uint64_t seed, int32_t cut, float* rgb,
                        float* queries) {
    Scene<float> S(*s);
    int64_t npix = camera_npix(*cam);
    int64_t n = npix * spp;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t p = 0; p < npix; ++p) {
        int view, row, col;
        camera_pixel(*cam, p, view, row, col);
        V3<float> acc(0.0f);
        Counters cnt;
        for (int sidx = 0; sidx < spp; ++sidx) {
            uint64_t pid = capture_path_id(p, sidx, npix);
            Rng rng(seed, pid, 0);
            V3<float> x, w;
            camera_ray(*cam, view, row, col, rng, x, w);
            PathHooks<float> hk;
            hk.cut = cut;
            acc += path_integrator_NEE(S, rng, x, w, false, cnt, &hk);
            V3<float> qx(0.0f), qw(0.0f, 0.0f, 1.0f), qW(0.0f);
            if (hk.queried) { qx = hk.qx; qw = hk.qw; qW = hk.qW; }
            float* q = queries + 3 * pid;
            q[0] = qx.x; q[1] = qx.y; q[2] = qx.z;
            q[3 * n + 0] = qw.x; q[3 * n + 1] = qw.y; q[3 * n + 2] = qw.z;
            q[6 * n + 0] = qW.x; q[6 * n + 1] = qW.y; q[6 * n + 2] = qW.z;
        }
        rgb[3 * p] += acc.x / (float)spp;
        rgb[3 * p + 1] += acc.y / (float)spp;
        rgb[3 * p + 2] += acc.z / (float)spp;
    }
}

void orc_train_samples(const orc_scene* s, const orc_camera* cam, int64_t n_paths, uint64_t seed, int32_t rec,
                       int32_t cut, float* samples) {
    Scene<float> S(*s);
    int64_t npix = (int64_t)cam->views * cam->height * cam->width;
    int64_t n = n_paths * rec;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n_paths; ++i) {
        Rng rng(seed, (uint64_t)i, 0);
        int64_t p = random_pixel(rng, npix);
        int view = (int)(p / ((int64_t)cam->height * cam->width));
        int rem = (int)(p % ((int64_t)cam->height * cam->width));
        V3<float> x, w;
        camera_ray(*cam, view, rem / cam->width, rem % cam->width, rng, x, w);
        PathHooks<float> hk;
        hk.rec = rec < 8 ? rec : 8;
        hk.cut = cut;
        Counters cnt;
        V3<float> R = path_integrator_NEE(S, rng, x, w, false, cnt, &hk);
        for (int k = 0; k < rec; ++k) {
            int64_t slot = i * rec + k;
            float* o = samples + 3 * slot;
            V3<float> px(0.0f), pw(0.0f, 0.0f, 1.0f), tg(NAN), wt(0.0f);
            if (k < hk.nrec) {
                px = hk.rx[k]; pw = hk.rw[k]; wt = hk.rW[k];
                V3<float> num = R - hk.rR[k];
                tg = V3<float>(num.x / wt.x, num.y / wt.y, num.z / wt.z);
            }
            o[0] = px.x; o[1] = px.y; o[2] = px.z;
            o[3 * n + 0] = pw.x; o[3 * n + 1] = pw.y; o[3 * n + 2] = pw.z;
            o[6 * n + 0] = tg.x; o[6 * n + 1] = tg.y; o[6 * n + 2] = tg.z;
            o[9 * n + 0] = wt.x; o[9 * n + 1] = wt.y; o[9 * n + 2] = wt.z;
        }
    }
}

void orc_capture_bw(const orc_scene* s, int32_t bw_mode, const orc_camera* cam, int32_t spp, uint64_t seed, const float* dL_drgb) {
    Scene<float> S(*s);
    int64_t npix = camera_npix(*cam);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t p = 0; p < npix; ++p) {
        int view, row, col;
        camera_pixel(*cam, p, view, row, col);
        V3<float> dL = V3<float>::load(dL_drgb + 3 * p) / (float)spp;
        for (int sidx = 0; sidx < spp; ++sidx) {
            Rng rng(seed, capture_path_id(p, sidx, npix), 0);
            V3<float> x, w;
            camera_ray(*cam, view, row, col, rng, x, w);
            radiance_bw(S, bw_mode, rng, x, w, dL);
        }
    }
}

}  // extern "C"
