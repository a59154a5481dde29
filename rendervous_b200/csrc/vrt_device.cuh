// vrt_device.cuh -- device building blocks of the volume hot path (sm_100a).
//
// Each function states the reference GLSL it re-implements.  Arithmetic keeps
// the reference's expression order where that order decides a branch (free
// flight, collision probability), so a path follows the same draws as the
// sequential definition.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "vrt_params.h"

namespace vrt {

// ------------------------------------------------------------------ Philox --
// Philox-4x32-10 (Salmon et al., SC'11), replacing the Tausworthe+LCG stream of
// the reference (include/randoms.h:6-59).  Draw k of stream s of path p is word
// k&3 of philox(seed, {k>>2, p_lo, s, p_hi}).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Each transmittance estimate draws from its own stream: the j-th fork of
// stream s is stream s + 2(j+1) (stream 0 is the path, stream 1 the DRT
// adjoint's branch stream).  Re-forking from a saved state replays a shadow
// ray exactly, which is what the reference's SAVE_SEED(before_transmittance)
// achieves with its single stream.
struct Rng {
    uint32_t k0, k1, plo, phi, stream, n, ntr;
    uint4 buf;

    __device__ __forceinline__ void init(uint64_t seed, uint64_t path, uint32_t s) {
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
        plo = (uint32_t)path; phi = (uint32_t)(path >> 32);
        stream = s; n = 0; ntr = 0;
    }
    __device__ __forceinline__ Rng fork() {
        Rng r = *this;
        r.stream = stream + 2u * (1u + ntr);
        r.n = 0;
        r.ntr = 0;
        ++ntr;
        return r;
    }
    __device__ __forceinline__ void refill() { buf = philox4x32_10(make_uint4(n >> 2, plo, stream, phi), k0, k1); }
    __device__ __forceinline__ uint32_t u32() {
        uint32_t j = n & 3u;
        if (j == 0) refill();
        uint32_t v = j == 0 ? buf.x : (j == 1 ? buf.y : (j == 2 ? buf.z : buf.w));
        ++n;
        return v;
    }
    // randoms.h:51-56: uintBitsToFloat(v & 0x7FFFFF | 0x3F800000) - 1, in [0,1)
    __device__ __forceinline__ float uniform() {
        return __uint_as_float((u32() & 0x007FFFFFu) | 0x3F800000u) - 1.0f;
    }
    __device__ __forceinline__ void advance() { (void)u32(); }  // randoms.h:35-41 advance_random
    // The DRTQ adjoint's scatter term of segment k (0: the primary ray's, k:
    // the one after the k-th scattering vertex): stream s + 1 of the path id
    // with k + 1 in bits 40-63 (path ids below 2^40, k + 1 below 2^24), so the
    // terms draw independently of one another and of the path.
    __device__ __forceinline__ Rng segment_stream(uint32_t k) const {
        Rng r = *this;
        r.phi = phi | ((k + 1u) << 8);
        r.stream = stream + 1u;
        r.n = 0;
        r.ntr = 0;
        return r;
    }
    // Position of the stream (draw index and forks taken) for replays.
    struct Pos { uint32_t n, ntr; };
    __device__ __forceinline__ Pos pos() const { return Pos{n, ntr}; }
    __device__ __forceinline__ void seek(Pos p) {
        n = p.n;
        ntr = p.ntr;
        if (n & 3u) refill();
    }
};

// ------------------------------------------------------------- float3 ops --
__device__ __forceinline__ float3 f3(float a) { return make_float3(a, a, a); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__device__ __forceinline__ float3 normalize(float3 a) { return a / sqrtf(dot(a, a)); }
__device__ __forceinline__ bool all_less(float3 a, float e) { return a.x < e && a.y < e && a.z < e; }
__device__ __forceinline__ float gmin(float a, float b) { return b < a ? b : a; }  // GLSL min
__device__ __forceinline__ float gmax(float a, float b) { return a < b ? b : a; }  // GLSL max
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float comp(float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__device__ __forceinline__ float3 ld3(const float* p) { return make_float3(p[0], p[1], p[2]); }

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.28318530717958647692f;

// ---------------------------------------------------------------- ray box --
// include/maths.h:28-38 ray_box_intersection (w components with |w|<=1e-6
// replaced by 1e-6) and :11-26 intersect_ray_box (tMin clamped at 0).
__device__ __forceinline__ float unpar(float w) { return fabsf(w) <= 0.000001f ? 0.000001f : w; }
__device__ __forceinline__ void ray_box_intersection(float3 x, float3 w, float3 bmin, float3 bmax, float& tMin, float& tMax) {
    w = make_float3(unpar(w.x), unpar(w.y), unpar(w.z));
    float3 cmin = (bmin - x) / w, cmax = (bmax - x) / w;
    tMin = gmax(gmax(gmin(cmin.x, cmax.x), gmin(cmin.y, cmax.y)), gmin(cmin.z, cmax.z));
    tMax = gmin(gmin(gmax(cmin.x, cmax.x), gmax(cmin.y, cmax.y)), gmax(cmin.z, cmax.z));
}
__device__ __forceinline__ bool intersect_ray_box(float3 x, float3 w, float3 bmin, float3 bmax, float& tMin, float& tMax) {
    ray_box_intersection(x, w, bmin, bmax, tMin, tMax);
    tMin = gmax(0.0f, tMin);
    return !(tMax <= tMin || tMax <= 0.0f);
}
// include/vr_boundary.h:1-11 over RayBoxIntersection
// A non-finite ray (NaN interval) counts as a miss, so no tracking loop starts on it.
__device__ __forceinline__ bool boundary(const DMedium& M, float3 x, float3 w, float& tMin, float& tMax) {
    ray_box_intersection(x, w, M.box_min, M.box_max, tMin, tMax);
    tMin = gmax(0.0f, tMin);
    return !(tMax < tMin) && tMax == tMax && tMin == tMin;
}

// ------------------------------------------------------------------ grids --
__device__ __forceinline__ float ldg(const float* p) { return __ldg(p); }

// Grid3D FORWARD (include/maps/grid3d.h:6-37): zero outside [0,1)^3, cell
// clamped to dim-1, weights from fract().  Channel 0 only.
__device__ __forceinline__ float grid_sigma(const DGrid& g, float3 nc) {
    if (nc.x < 0.0f || nc.y < 0.0f || nc.z < 0.0f || nc.x >= 1.0f || nc.y >= 1.0f || nc.z >= 1.0f) return 0.0f;
    const int dx = g.W - 1, dy = g.H - 1, dz = g.D - 1;
    float gx = nc.x * (float)dx, gy = nc.y * (float)dy, gz = nc.z * (float)dz;
    float ax = gx - floorf(gx), ay = gy - floorf(gy), az = gz - floorf(gz);
    int px = min(max((int)gx, 0), dx - 1), py = min(max((int)gy, 0), dy - 1), pz = min(max((int)gz, 0), dz - 1);
    const float* b = g.data + (pz * g.sD + py * g.sH + px * g.sW);
    float v000 = ldg(b), v100 = ldg(b + g.sW), v010 = ldg(b + g.sH), v110 = ldg(b + g.sH + g.sW);
    float v001 = ldg(b + g.sD), v101 = ldg(b + g.sD + g.sW), v011 = ldg(b + g.sD + g.sH), v111 = ldg(b + g.sD + g.sH + g.sW);
    float bx = 1.0f - ax, by = 1.0f - ay, bz = 1.0f - az;
    float o = 0.0f;
    o += v000 * (bx * by * bz);
    o += v100 * (ax * by * bz);
    o += v010 * (bx * ay * bz);
    o += v110 * (ax * ay * bz);
    o += v001 * (bx * by * az);
    o += v101 * (ax * by * az);
    o += v011 * (bx * ay * az);
    o += v111 * (ax * ay * az);
    return o;
}

__device__ __forceinline__ float3 normalized(const DMedium& M, float3 x) {
    return make_float3((x.x - M.bmin.x) * M.inv_bsize.x, (x.y - M.bmin.y) * M.inv_bsize.y, (x.z - M.bmin.z) * M.inv_bsize.z);
}
// Per-thread work tally: free-flight steps, sigma lookups (8 node gathers
// each), atomic adds, albedo lookups and bytes of the NEE_DS collision log
// written or read.  Kept in registers, summed per warp.
struct Tally {
    uint32_t steps = 0, lookups = 0, reds = 0, albedo = 0, logb = 0;
};

__device__ __forceinline__ float sigma(const DMedium& M, float3 x, Tally& tl) {
    ++tl.lookups;
    return grid_sigma(M.sigma, normalized(M, x));
}

// Grid3D BACKWARD (include/maps/grid3d.h:39-75): 8 atomic adds per channel.
__device__ __forceinline__ void red_add(float* p, float v) { atomicAdd(p, v); }

// Two adjacent floats added by one vector atomic (sm_90+) when the first is
// 8-byte aligned, else by two scalar ones; each component is still its own
// atomic add of the same value.
__device__ __forceinline__ void red_add2(float* p, float a, float b) {
    if ((reinterpret_cast<uintptr_t>(p) & 7u) == 0u) {
        atomicAdd(reinterpret_cast<float2*>(p), make_float2(a, b));
    } else {
        atomicAdd(p, a);
        atomicAdd(p + 1, b);
    }
}
// Three adjacent floats (one node's channels): a vector pair and a scalar.
__device__ __forceinline__ void red_add3(float* p, float a, float b, float c) {
    if ((reinterpret_cast<uintptr_t>(p) & 7u) == 0u) {
        atomicAdd(reinterpret_cast<float2*>(p), make_float2(a, b));
        atomicAdd(p + 2, c);
    } else {
        atomicAdd(p, a);
        atomicAdd(reinterpret_cast<float2*>(p + 1), make_float2(b, c));
    }
}

__device__ __forceinline__ void grid_scatter(const DGrid& g, float3 nc, const float* dout, int C) {
    if (!g.grad) return;
    if (nc.x < 0.0f || nc.y < 0.0f || nc.z < 0.0f || nc.x >= 1.0f || nc.y >= 1.0f || nc.z >= 1.0f) return;
    const int dx = g.W - 1, dy = g.H - 1, dz = g.D - 1;
    float gx = nc.x * (float)dx, gy = nc.y * (float)dy, gz = nc.z * (float)dz;
    float ax = gx - floorf(gx), ay = gy - floorf(gy), az = gz - floorf(gz);
    int px = min(max((int)gx, 0), dx - 1), py = min(max((int)gy, 0), dy - 1), pz = min(max((int)gz, 0), dz - 1);
    float* b = g.grad + (pz * g.sD + py * g.sH + px * g.sW);
    float bx = 1.0f - ax, by = 1.0f - ay, bz = 1.0f - az;
    if (C == 1 && g.sW == 1) {  // x-neighbours adjacent: the four x-pairs as vector pairs where aligned
        const float d = dout[0];
        red_add2(b, d * bx * by * bz, d * ax * by * bz);
        red_add2(b + g.sH, d * bx * ay * bz, d * ax * ay * bz);
        red_add2(b + g.sD, d * bx * by * az, d * ax * by * az);
        red_add2(b + g.sD + g.sH, d * bx * ay * az, d * ax * ay * az);
        return;
    }
    if (C == 3) {  // a node's three channels adjacent (channel stride 1)
        const float d0 = dout[0], d1 = dout[1], d2 = dout[2];
        // the same products, in the same order, as the per-channel form below
#define VRT_CORNER(o, fx, fy, fz) red_add3(b + (o), d0 * fx * fy * fz, d1 * fx * fy * fz, d2 * fx * fy * fz)
        VRT_CORNER(0, bx, by, bz);
        VRT_CORNER(g.sW, ax, by, bz);
        VRT_CORNER(g.sH, bx, ay, bz);
        VRT_CORNER(g.sH + g.sW, ax, ay, bz);
        VRT_CORNER(g.sD, bx, by, az);
        VRT_CORNER(g.sD + g.sW, ax, by, az);
        VRT_CORNER(g.sD + g.sH, bx, ay, az);
        VRT_CORNER(g.sD + g.sH + g.sW, ax, ay, az);
#undef VRT_CORNER
        return;
    }
    for (int i = 0; i < C; ++i) {
        float d = dout[i];
        red_add(b + i, d * bx * by * bz);
        red_add(b + g.sW + i, d * ax * by * bz);
        red_add(b + g.sH + i, d * bx * ay * bz);
        red_add(b + g.sH + g.sW + i, d * ax * ay * bz);
        red_add(b + g.sD + i, d * bx * by * az);
        red_add(b + g.sD + g.sW + i, d * ax * by * az);
        red_add(b + g.sD + g.sH + i, d * bx * ay * az);
        red_add(b + g.sD + g.sH + g.sW + i, d * ax * ay * az);
    }
}
__device__ __forceinline__ void sigma_bw(const DMedium& M, float3 x, float dL, Tally& tl) {
    if (dL == 0.0f) return;
    tl.reds += 8;
    grid_scatter(M.sigma, normalized(M, x), &dL, 1);
}

// Grid3D lookup of a C == 1 (promoted to 3) or C == 3 grid at normalized
// coordinates nc (include/maps/grid3d.h:6-37): zero outside [0, 1)^3.
__device__ __forceinline__ float3 grid_rgb(const DGrid& g, float3 nc) {
    if (nc.x < 0.0f || nc.y < 0.0f || nc.z < 0.0f || nc.x >= 1.0f || nc.y >= 1.0f || nc.z >= 1.0f) return f3(0.0f);
    const int dx = g.W - 1, dy = g.H - 1, dz = g.D - 1;
    float gx = nc.x * (float)dx, gy = nc.y * (float)dy, gz = nc.z * (float)dz;
    float ax = gx - floorf(gx), ay = gy - floorf(gy), az = gz - floorf(gz);
    int px = min(max((int)gx, 0), dx - 1), py = min(max((int)gy, 0), dy - 1), pz = min(max((int)gz, 0), dz - 1);
    const float* b = g.data + (pz * g.sD + py * g.sH + px * g.sW);
    float bx = 1.0f - ax, by = 1.0f - ay, bz = 1.0f - az;
    const int off[8] = {0, g.sW, g.sH, g.sH + g.sW, g.sD, g.sD + g.sW, g.sD + g.sH, g.sD + g.sH + g.sW};
    const float wt[8] = {bx * by * bz, ax * by * bz, bx * ay * bz, ax * ay * bz,
                         bx * by * az, ax * by * az, bx * ay * az, ax * ay * az};
    if (g.C == 1) {
        float o = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) o += ldg(b + off[k]) * wt[k];
        return f3(o);
    }
    float3 o = f3(0.0f);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float* p = b + off[k];
        o.x += ldg(p) * wt[k];
        o.y += ldg(p + 1) * wt[k];
        o.z += ldg(p + 2) * wt[k];
    }
    return o;
}
// Adjoint of grid_rgb (a C == 1 grid receives the channel sum).
__device__ __forceinline__ void grid_rgb_bw(const DGrid& g, float3 nc, float3 dL) {
    if (g.C == 1) {
        float s = dL.x + dL.y + dL.z;
        grid_scatter(g, nc, &s, 1);
    } else {
        float d[3] = {dL.x, dL.y, dL.z};
        grid_scatter(g, nc, d, 3);
    }
}

// Albedo: const or Grid3D with C 1 (promoted to 3) or 3 (include/vr_scattering_albedo.h).
__device__ __forceinline__ float3 albedo(const DMedium& M, float3 x, Tally& tl) {
    if (!M.albedo_is_grid) return M.albedo_const;
    ++tl.albedo;
    return grid_rgb(M.albedo, normalized(M, x));
}
__device__ __forceinline__ void albedo_bw(const DMedium& M, float3 x, float3 dL, Tally& tl) {
    if (!M.albedo_is_grid || !M.albedo.grad) return;
    tl.reds += 8 * M.albedo.C;
    grid_rgb_bw(M.albedo, normalized(M, x), dL);
}

// Emission of the collision integrators' exitance (include/vr_emission.h):
// const, or a Grid3D (C 1 or 3) over sigma's box.
__device__ __forceinline__ float3 emission_at(const DMedium& M, float3 x) {
    if (!M.emission_is_grid) return M.emission;
    return grid_rgb(M.emission_grid, normalized(M, x));
}
__device__ __forceinline__ void emission_bw(const DMedium& M, float3 x, float3 dL, Tally& tl) {
    if (!M.emission_is_grid || !M.emission_grid.grad) return;
    tl.reds += 8 * M.emission_grid.C;
    grid_rgb_bw(M.emission_grid, normalized(M, x), dL);
}

// ------------------------------------------------------------- majorant --
// include/vr_majorant.h:1-7.  Mode 0: the constant [max sigma, 1e6]
// (_objects.py:96-101).  Mode 1 (no reference counterpart): a brick grid; the
// query returns the brick's bound and the distance to leave the brick.  A
// point within 1e-4 brick widths of a face is assigned to the brick that w
// enters, so a ray parked on a face always makes progress.
// Outside the grid's box the bound is 0 (Grid3D is zero there) and the
// distance is the one to (re-)enter the box, or 1e6 when w leaves it.
__device__ __forceinline__ float majorant(const DMedium& M, float3 x, float3 w, float& md) {
    if (M.maj_mode == 0) { md = 1000000.0f; return M.gmaj; }
    const float inf = __int_as_float(0x7f800000);
    const int Md[3] = {M.Mx, M.My, M.Mz};
    bool inside = true;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float q = (comp(x, i) - comp(M.bmin, i)) * comp(M.maj_scale, i);
        if (!(q >= 0.0f && q <= (float)Md[i])) inside = false;
    }
    if (!inside) {
        float tn = -inf, tf = inf;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            float q = (comp(x, i) - comp(M.bmin, i)) * comp(M.maj_scale, i);
            float v = comp(w, i) * comp(M.maj_scale, i);
            if (v != 0.0f) {
                float rv = __frcp_rn(v);
                float a = (0.0f - q) * rv, b = ((float)Md[i] - q) * rv;
                tn = gmax(tn, gmin(a, b));
                tf = gmin(tf, gmax(a, b));
            } else if (!(q >= 0.0f && q <= (float)Md[i])) {
                tn = inf;
            }
        }
        md = (tn < tf && tn > 0.0f) ? gmax(tn, 1e-6f) : 1000000.0f;
        return 0.0f;
    }
    int c[3];
    float dist = inf;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float xi = comp(x, i), wi = comp(w, i);
        float q = (xi - comp(M.bmin, i)) * comp(M.maj_scale, i);
        float nudge = wi > 0.0f ? 1e-4f : (wi < 0.0f ? -1e-4f : 0.0f);
        int ci = (int)floorf(q + nudge);
        ci = min(max(ci, 0), Md[i] - 1);
        c[i] = ci;
        float v = wi * comp(M.maj_scale, i);
        float rv = __frcp_rn(v);  // face distances use a correctly rounded reciprocal
        float di = v > 0.0f ? ((float)(ci + 1) - q) * rv : (v < 0.0f ? ((float)ci - q) * rv : __int_as_float(0x7f800000));
        dist = gmin(dist, di);
    }
    md = gmax(dist, 1e-6f);
    return __ldg(M.maj + ((c[2] * M.My + c[1]) * M.Mx + c[0]));
}

// ---------------------------------------------------------- directions --
// include/randoms.h:144-162 createOrthoBasis / randomDirection
__device__ __forceinline__ void ortho_basis(float3 N, float3& t, float3& b) {
    float sign = N.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sign + N.z);
    float bb = N.x * N.y * a;
    t = make_float3(1.0f + sign * N.x * N.x * a, sign * bb, -sign * N.x);
    b = make_float3(bb, sign + N.y * N.y * a, -N.y);
}
__device__ __forceinline__ float3 random_direction_y(Rng& rng) {
    float r1 = rng.uniform();
    float r2 = rng.uniform() * 2.0f - 1.0f;
    float st = sqrtf(gmax(0.0f, 1.0f - r2 * r2));
    float ang = kTwoPi * r1;
    float x = cosf(ang) * st, y = sinf(ang) * st;
    // basis of D = (0,1,0): t0 = (1,0,0), t1 = (0,0,-1)
    float3 t0, t1;
    ortho_basis(make_float3(0.0f, 1.0f, 0.0f), t0, t1);
    return t0 * x + t1 * y + make_float3(0.0f, 1.0f, 0.0f) * r2;
}
// include/scattering_AD.h:4-19 hg_phase_sample, :37-45 hg_phase_eval
__device__ __forceinline__ float3 hg_phase_sample(Rng& rng, float3 w_in, float g) {
    float phi = rng.uniform() * 2.0f * kPi;
    float xi = rng.uniform();
    float g2 = g * g;
    float t = (1.0f - g2) / (1.0f - g + 2.0f * g * xi);
    float inv = (0.5f / g) * ((1.0f + g2) - t * t);
    float ct = fabsf(g) < 0.001f ? 2.0f * xi - 1.0f : inv;
    float st = sqrtf(gmax(0.0f, 1.0f - ct * ct));
    float3 t0, t1;
    ortho_basis(w_in, t0, t1);
    return st * sinf(phi) * t0 + st * cosf(phi) * t1 + ct * w_in;
}
__device__ __forceinline__ float hg_phase_eval(float c, float g) {
    if (fabsf(g) < 0.001f) return 0.25f / kPi;
    float g2 = g * g;
    return 0.25f / kPi * (1.0f - g2) / powf(1.0f + g2 - 2.0f * g * c, 1.5f);
}
// include/vr_phase.h over HGPhase (_maps.py:4436-4460) or pure HG
__device__ __forceinline__ float phase(const DMedium& M, float3 w, float3 wo) {
    float c = dot(w, wo);
    if (M.phase_mode == 1) return mixf(hg_phase_eval(c, M.g), hg_phase_eval(c, M.g / 5.0f), 0.2f);
    return hg_phase_eval(c, M.g);
}
// include/vr_phase_sampler.h over VHGPhaseSampler (_maps.py:4463-4484) or pure HG; weight 1
__device__ __forceinline__ float3 phase_sample(const DMedium& M, Rng& rng, float3 w) {
    float g = M.g;
    if (M.phase_mode == 1) {
        if (rng.uniform() < 0.8f) g = g / 5.0f;
    }
    return hg_phase_sample(rng, w, g);
}
// ------------------------------------------------------------ environment --
// include/maths.h:172-178 dir2xr: equirectangular coordinates in [-1, 1]^2.
__device__ __forceinline__ float2 dir2xr(float3 w) {
    if (w.x == 0.0f && w.z == 0.0f) w.x += 0.0000001f;
    const float x = atan2f(w.x, w.z) * (1.0f / kPi);
    const float y = -2.0f * asinf(fminf(fmaxf(w.y, -1.0f), 1.0f)) * (1.0f / kPi);
    return make_float2(x, y);
}
// The environment radiance towards w: the constant env, or
// Image2D(env image).after(xr_projection) (_objects.py:165-172,
// include/maps/image2d.h:1-26 with its default box [-1, 1]^2: clamped
// coordinates, bilinear over pixel centres, clamped pixel indices).
__device__ __forceinline__ float3 env_radiance(const DMedium& M, float3 w) {
    if (M.env_mode == 0) return M.env;
    const float2 c = dir2xr(w);
    const float nx = fminf(fmaxf((c.x - (-1.0f)) * 0.5f, 0.0f), 1.0f);
    const float ny = fminf(fmaxf((c.y - (-1.0f)) * 0.5f, 0.0f), 1.0f);
    const float gx = nx * (float)M.env_w - 0.5f, gy = ny * (float)M.env_h - 0.5f;
    const float fx = floorf(gx), fy = floorf(gy);
    const int px = (int)fx, py = (int)fy;
    const float ax = gx - fx, ay = gy - fy;
    const int x0 = min(max(px, 0), M.env_w - 1), x1 = min(max(px + 1, 0), M.env_w - 1);
    const int y0 = min(max(py, 0), M.env_h - 1), y1 = min(max(py + 1, 0), M.env_h - 1);
    const float* r0 = M.env_img + 3 * (y0 * M.env_w);
    const float* r1 = M.env_img + 3 * (y1 * M.env_w);
    float3 o;
    o.x = mixf(mixf(ldg(r0 + 3 * x0), ldg(r0 + 3 * x1), ax), mixf(ldg(r1 + 3 * x0), ldg(r1 + 3 * x1), ax), ay);
    o.y = mixf(mixf(ldg(r0 + 3 * x0 + 1), ldg(r0 + 3 * x1 + 1), ax), mixf(ldg(r1 + 3 * x0 + 1), ldg(r1 + 3 * x1 + 1), ax), ay);
    o.z = mixf(mixf(ldg(r0 + 3 * x0 + 2), ldg(r0 + 3 * x1 + 2), ax), mixf(ldg(r1 + 3 * x0 + 2), ldg(r1 + 3 * x1 + 2), ax), ay);
    return o;
}
// include/randoms.h:186-199 randomDirection(alpha0, alpha1, beta0, beta1):
// azimuth uniform in [alpha0, alpha1], cos of the polar angle (about +y)
// uniform between cos(beta0) and cos(beta1).
__device__ __forceinline__ float3 random_direction_range(Rng& rng, float a0, float a1, float b0, float b1) {
    const float r1 = rng.uniform() * (a1 - a0) + a0;
    const float r2 = cosf(b0) - rng.uniform() * (cosf(b0) - cosf(b1));
    const float s = sqrtf(gmax(0.0f, 1.0f - r2 * r2));
    return make_float3(sinf(r1) * s, r2, cosf(r1) * s);
}
// include/vr_environment_sampler.h over _functionsampler(point sampler, environment)
// (_maps.py:2552-2585): [E(w) * weight, w] with the point sampler
//   UniformDirectionSampler (include/maps/uniform_direction_sampler.h:1-5): weight 4 pi, or
//   XRQuadtreeRandomDirection (_maps.py:2494-2549): a pixel of the image drawn
//   down the probability quadtree with one uniform (node k's children at
//   4k + 1 .. 4k + 4, child c = 2 * (lower half) + (right half)), then a
//   direction uniform in its solid angle; weight = pixel solid angle / p.
__device__ __forceinline__ float3 environment_sample(const DMedium& M, Rng& rng, float3& wo) {
    if (M.env_sampler == 0) {
        wo = random_direction_y(rng);
        return env_radiance(M, wo) * (4.0f * kPi);
    }
    float sel = rng.uniform();
    int node = 0;
    float p0x = 0.0f, p0y = 0.0f, p1x = 1.0f, p1y = 1.0f, prob = 1.0f;
    for (int i = 0; i < M.env_levels; ++i) {
        const float* d = M.env_qt + node * 4;
        int child = 3;
        prob = ldg(d + 3);
        for (int c = 0; c < 3; ++c) {
            const float dc = ldg(d + c);
            if (sel < dc) {
                child = c;
                prob = dc;
                break;
            }
            sel -= dc;
        }
        const float xmed = (p1x + p0x) / 2.0f, ymed = (p1y + p0y) / 2.0f;
        if (child % 2 == 0) p1x = xmed; else p0x = xmed;
        if (child / 2 == 0) p1y = ymed; else p0y = ymed;
        node = node * 4 + 1 + child;
    }
    const float pixel_area = 2.0f * kPi * (cosf(p0y * kPi) - cosf(p1y * kPi)) / (float)(1 << M.env_levels);
    const float weight = pixel_area / gmax(0.000000001f, prob);
    wo = random_direction_range(rng, (p0x * 2.0f - 1.0f) * kPi, (p1x * 2.0f - 1.0f) * kPi, p0y * kPi, p1y * kPi);
    return env_radiance(M, wo) * weight;
}

// The path walks are compiled twice: with IMG false they handle only the
// constant environment under the uniform direction sampler (the same values as
// env_radiance / environment_sample give for it), which keeps the image lookup
// and the quadtree descent out of the kernels that do not need them.
template <bool IMG>
__device__ __forceinline__ float3 env_radiance_t(const DMedium& M, float3 w) {
    return IMG ? env_radiance(M, w) : M.env;
}
template <bool IMG>
__device__ __forceinline__ float3 environment_sample_t(const DMedium& M, Rng& rng, float3& wo) {
    if (IMG) return environment_sample(M, rng, wo);
    wo = random_direction_y(rng);
    return M.env * (4.0f * kPi);
}

// ---------------------------------------------------------------- camera --
// include/maps/sensor_perspective_camera.h:1-27
__device__ __forceinline__ void camera_ray(const DCamera& C, int view, int row, int col, Rng& rng, float3& x, float3& w) {
    const float* p = C.poses + 9 * view;
    float3 o = ld3(p), dd = ld3(p + 3), n = ld3(p + 6);
    float sx_ = 0.5f, sy_ = 0.5f;
    if (C.jittered) { sx_ = rng.uniform(); sy_ = rng.uniform(); }
    float sx = (((float)col + sx_) * 2.0f - (float)C.width) * C.znear / (float)C.height;
    float sy = (((float)row + sy_) * 2.0f - (float)C.height) * C.znear / (float)C.height;
    float sz = C.znear / tanf(C.fov * 0.5f);
    float3 zaxis = normalize(dd);
    float3 xaxis = normalize(cross(n, zaxis));
    float3 yaxis = cross(zaxis, xaxis);
    w = xaxis * sx + yaxis * sy + zaxis * sz;
    x = o + w;
    w = normalize(w);
}

// Primary ray of capture pixel px (0 <= px < npix): pixels of all views in
// raster order, or entry px of a sensors batch (the capture kernel's index
// decoding, _maps.py:560-577).  A sensors entry outside the camera sets the
// invalid-argument bit and returns false (the path adds nothing).
__device__ __forceinline__ bool camera_pixel_ray(const DCamera& C, long long px, Rng& rng, float3& x, float3& w,
                                                 uint32_t* status) {
    int view, row, col;
    if (C.sensors) {
        const long long v = C.sensors[3 * px], r = C.sensors[3 * px + 1], c = C.sensors[3 * px + 2];
        if (v < 0 || v >= C.views || r < 0 || r >= C.height || c < 0 || c >= C.width) {
            if (status) atomicOr(status, 1u << 1);
            x = make_float3(0.0f, 0.0f, 0.0f);
            w = make_float3(__int_as_float(0x7fc00000), 0.0f, 0.0f);  // a NaN ray misses the medium
            return false;
        }
        view = (int)v; row = (int)r; col = (int)c;
    } else {
        const long long hw = (long long)C.height * C.width;
        view = (int)(px / hw);
        const int rem = (int)(px - (long long)view * hw);
        row = rem / C.width;
        col = rem % C.width;
    }
    camera_ray(C, view, row, col, rng, x, w);
    return true;
}

// ------------------------------------------------------------ diagnostics --
__device__ __forceinline__ void raise_status(uint32_t* status, int code) {
    if (status) atomicOr(status, 1u << code);
}

}  // namespace vrt
