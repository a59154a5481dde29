// vrt_fp64.cu -- the plain NEE path tracer in FP64 (sm_100a).
//
// The high-accuracy estimate the radiance cache's error is measured against
// (no reference counterpart: the reference renders in FP32 only).  It is the
// path integrator of include/vr_path_integrator_NEE.h:1-66 with the
// directional light and the bounce cap of the FP32 kernels, every quantity in
// double: grid values are read as float and widened, the Philox draws are the
// FP32 tracer's (a float uniform widened), and the arithmetic follows the
// CPU restatement instantiated on double formula for formula -- division-form
// free flights, correctly rounded reciprocals in the brick walk -- so the two
// agree path for path to rounding.  One path per thread, grid-stride; pixel
// sums in double.  Media: sigma Grid3D, albedo const or Grid3D, constant
// emission and environment (uniform-sphere NEE), optional sun, HG or the
// reference's VHG mixture, constant or brick majorant, ratio- or
// delta-tracking shadow rays.
#include <cuda_runtime.h>

#include "../../include/vrt.h"
#include "vrt_device.cuh"
#include "vrt_internal.h"

namespace vrt {
namespace {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 d3(double a, double b, double c) { return D3{a, b, c}; }
__device__ __forceinline__ D3 d3(float3 v) { return D3{(double)v.x, (double)v.y, (double)v.z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ D3 operator*(D3 a, D3 b) { return d3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ D3 operator/(D3 a, D3 b) { return d3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return d3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ D3 operator/(D3 a, double s) { return d3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ double dotd(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 crossd(D3 a, D3 b) {
    return d3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__device__ __forceinline__ D3 normd(D3 a) { return a / sqrt(dotd(a, a)); }
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }  // GLSL min
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }  // GLSL max
__device__ __forceinline__ double cmp(D3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__device__ __forceinline__ double cmp(float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__device__ __forceinline__ double uni(Rng& r) { return (double)r.uniform(); }

constexpr double kPiD = 3.14159265358979323846;

// include/maths.h:28-38 and vr_boundary.h:1-11 (a NaN interval is a miss)
__device__ __forceinline__ bool boundary_d(const DMedium& M, D3 x, D3 w, double& tMin, double& tMax) {
    const double e = 0.000001;
    const D3 wu = d3(fabs(w.x) <= e ? e : w.x, fabs(w.y) <= e ? e : w.y, fabs(w.z) <= e ? e : w.z);
    const D3 cmin = (d3(M.box_min) - x) / wu, cmax = (d3(M.box_max) - x) / wu;
    tMin = dmax(dmax(dmin(cmin.x, cmax.x), dmin(cmin.y, cmax.y)), dmin(cmin.z, cmax.z));
    tMax = dmin(dmin(dmax(cmin.x, cmax.x), dmax(cmin.y, cmax.y)), dmax(cmin.z, cmax.z));
    tMin = dmax(0.0, tMin);
    return !(tMax < tMin) && tMax == tMax && tMin == tMin;
}

// Grid3D lookup (include/maps/grid3d.h:6-37) at x, zero outside the box
__device__ __forceinline__ void grid_d(const DMedium& M, const DGrid& g, D3 x, double* out) {
    const D3 nc = d3((x.x - (double)M.bmin.x) * (double)M.inv_bsize.x, (x.y - (double)M.bmin.y) * (double)M.inv_bsize.y,
                     (x.z - (double)M.bmin.z) * (double)M.inv_bsize.z);
    for (int i = 0; i < g.C; ++i) out[i] = 0.0;
    if (nc.x < 0.0 || nc.y < 0.0 || nc.z < 0.0 || nc.x >= 1.0 || nc.y >= 1.0 || nc.z >= 1.0) return;
    const int dx = g.W - 1, dy = g.H - 1, dz = g.D - 1;
    const D3 gc = d3(nc.x * dx, nc.y * dy, nc.z * dz);
    const D3 a = d3(gc.x - floor(gc.x), gc.y - floor(gc.y), gc.z - floor(gc.z));
    const int px = min(max((int)gc.x, 0), dx - 1), py = min(max((int)gc.y, 0), dy - 1), pz = min(max((int)gc.z, 0), dz - 1);
    for (int k = 0; k < 8; ++k) {
        const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
        const double wx = ox ? a.x : 1.0 - a.x, wy = oy ? a.y : 1.0 - a.y, wz = oz ? a.z : 1.0 - a.z;
        const double wt = wx * wy * wz;
        const float* src = g.data + ((pz + oz) * g.sD + (py + oy) * g.sH + (px + ox) * g.sW);
        for (int i = 0; i < g.C; ++i) out[i] += (double)__ldg(src + i) * wt;
    }
}
__device__ __forceinline__ double sigma_d(const DMedium& M, D3 x) {
    double v;
    grid_d(M, M.sigma, x, &v);
    return v;
}
__device__ __forceinline__ D3 albedo_d(const DMedium& M, D3 x) {
    if (!M.albedo_is_grid) return d3(M.albedo_const);
    double v[3];
    grid_d(M, M.albedo, x, v);
    return M.albedo.C == 1 ? d3(v[0], v[0], v[0]) : d3(v[0], v[1], v[2]);
}

// Majorant bricks along a segment (the FP32 walk's rules in double)
struct BrickWalkD {
    bool live = false;
    int c[3], st[3];
    double tn[3], dt[3], t, m;
    __device__ __forceinline__ double lookup(const DMedium& M) const {
        const int Md[3] = {M.Mx, M.My, M.Mz};
        for (int i = 0; i < 3; ++i)
            if (c[i] < 0 || c[i] >= Md[i]) return 0.0;
        return (double)__ldg(M.maj + ((c[2] * M.My + c[1]) * M.Mx + c[0]));
    }
    __device__ __forceinline__ void init(const DMedium& M, D3 x, D3 w) {
        live = true;
        t = 0.0;
        const double inf = __longlong_as_double(0x7ff0000000000000ll);
        for (int i = 0; i < 3; ++i) {
            const double q = (cmp(x, i) - cmp(M.bmin, i)) * cmp(M.maj_scale, i);
            const double dq = cmp(w, i) * cmp(M.maj_scale, i);
            if (dq > 0.0) {
                c[i] = (int)floor(q + 1e-4); st[i] = 1;
                const double rv = 1.0 / dq;
                tn[i] = ((double)(c[i] + 1) - q) * rv; dt[i] = rv;
            } else if (dq < 0.0) {
                c[i] = (int)floor(q - 1e-4); st[i] = -1;
                const double rv = 1.0 / dq;
                tn[i] = ((double)c[i] - q) * rv; dt[i] = -rv;
            } else {
                c[i] = (int)floor(q); st[i] = 0; tn[i] = inf; dt[i] = inf;
            }
        }
        m = lookup(M);
        if (never_enters(M)) tn[0] = tn[1] = tn[2] = inf;  // a segment that never reaches the grid: no face
    }
    __device__ __forceinline__ int axis() const { return (tn[0] <= tn[1] && tn[0] <= tn[2]) ? 0 : (tn[1] <= tn[2] ? 1 : 2); }
    __device__ __forceinline__ bool never_enters(const DMedium& M) const {
        const int Md[3] = {M.Mx, M.My, M.Mz};
        for (int i = 0; i < 3; ++i)
            if ((c[i] < 0 && st[i] <= 0) || (c[i] >= Md[i] && st[i] >= 0)) return true;
        return false;
    }
    __device__ __forceinline__ double query(const DMedium& M, D3 x, D3 w, double& md) {
        if (M.maj_mode == 0) { md = 1000000.0; return (double)M.gmaj; }
        if (!live) init(M, x, w);
        md = tn[axis()] - t;
        return m;
    }
    __device__ __forceinline__ void advance(const DMedium& M) {
        if (!live) return;
        const int a = axis();
        t = tn[a];
        tn[a] += dt[a];
        c[a] += st[a];
        m = lookup(M);
    }
};
struct FlightD {
    double tau = -1.0;
    BrickWalkD bk;
    __device__ __forceinline__ double sample(Rng& r) {
        if (tau < 0.0) tau = -log(1.0 - uni(r));
        return tau;
    }
    __device__ __forceinline__ void cross(double m, double md) { tau -= m * md; }
    __device__ __forceinline__ void used() { tau = -1.0; }
};

// include/vr_transmittance_RT.h:1-49 / _DT.h:1-28 in double
__device__ double transmittance_d(const DMedium& M, Rng& rng, D3 x, D3 w, uint32_t* status) {
    Rng r = rng.fork();
    double tMin, tMax;
    if (!boundary_d(M, x, w, tMin, tMax)) return 1.0;
    x = x + w * tMin;
    double d = tMax - tMin;
    double Tr = 1.0;
    FlightD ff;
    for (int it = 0; it < (1 << 24); ++it) {
        double md;
        const double maj = dmax(0.0000001, ff.bk.query(M, x, w, md));
        if (M.tr_mode == 0) {
            const double t = ff.sample(r) / maj;
            if (md < d && t > md) { x = x + w * md; d -= md; ff.cross(maj, md); ff.bk.advance(M); continue; }
            ff.used();
            const double dt = dmin(t, dmin(d, md));
            ff.bk.t += dt;
            x = x + w * dt;
            d -= dt;
            if (d <= 0.0000001) return Tr;
            Tr *= (1.0 - sigma_d(M, x) / maj);
            if (Tr < 0.01) {
                if (uni(r) < 1.0 - Tr) return 0.0;
                Tr = 1.0;
            }
        } else {
            const double dt = ff.sample(r) / maj;
            const double t = dmin(md, dt);
            x = x + w * t;
            d -= t;
            if (d <= 0.0000001) return 1.0;
            if (dt > md) { ff.cross(maj, md); ff.bk.advance(M); continue; }
            ff.used();
            ff.bk.t += t;
            if (uni(r) < sigma_d(M, x) / maj) return 0.0;
        }
    }
    raise_status(status, 4);
    return Tr;
}

// include/randoms.h:144-162 createOrthoBasis, include/scattering_AD.h:4-52
__device__ __forceinline__ void ortho_d(D3 N, D3& t, D3& b) {
    const double sign = N.z >= 0.0 ? 1.0 : -1.0;
    const double a = -1.0 / (sign + N.z);
    const double bb = N.x * N.y * a;
    t = d3(1.0 + sign * N.x * N.x * a, sign * bb, -sign * N.x);
    b = d3(bb, sign + N.y * N.y * a, -N.y);
}
__device__ __forceinline__ D3 random_direction_d(Rng& rng, D3 D) {
    const double r1 = uni(rng);
    const double r2 = uni(rng) * 2.0 - 1.0;
    const double ang = 2.0 * kPiD * r1;
    const double st = sqrt(dmax(0.0, 1.0 - r2 * r2));
    D3 t0, t1;
    ortho_d(D, t0, t1);
    return t0 * (cos(ang) * st) + t1 * (sin(ang) * st) + D * r2;
}
__device__ __forceinline__ D3 hg_sample_d(Rng& rng, D3 w_in, double g) {
    const double phi = uni(rng) * 2.0 * kPiD;
    const double xi = uni(rng);
    const double g2 = g * g, omg2 = 1.0 - g2, opg2 = 1.0 + g2, o2g = 0.5 / g;
    const double t = omg2 / (1.0 - g + 2.0 * g * xi);
    const double inv = o2g * (opg2 - t * t);
    const double ct = fabs(g) < 0.001 ? 2.0 * xi - 1.0 : inv;
    const double st = sqrt(dmax(0.0, 1.0 - ct * ct));
    D3 t0, t1;
    ortho_d(w_in, t0, t1);
    return st * sin(phi) * t0 + st * cos(phi) * t1 + ct * w_in;
}
__device__ __forceinline__ double hg_eval_d(double c, double g) {
    if (fabs(g) < 0.001) return 0.25 / kPiD;
    const double g2 = g * g;
    return 0.25 / kPiD * (1.0 - g2) / pow(1.0 + g2 - 2.0 * g * c, 1.5);
}
__device__ __forceinline__ double phase_d(const DMedium& M, D3 w, D3 wo) {
    const double g = (double)M.g, c = dotd(w, wo);
    if (M.phase_mode == 1) {
        const double a = hg_eval_d(c, g), b = hg_eval_d(c, g / 5.0);
        return a * (1.0 - 0.2) + b * 0.2;
    }
    return hg_eval_d(c, g);
}
__device__ __forceinline__ D3 phase_sample_d(const DMedium& M, Rng& rng, D3 w) {
    double g = (double)M.g;
    if (M.phase_mode == 1 && uni(rng) < 0.8) g = g / 5.0;
    return hg_sample_d(rng, w, g);
}

// include/maps/sensor_perspective_camera.h:1-27 in double
__device__ __forceinline__ void camera_d(const DCamera& C, long long px, Rng& rng, D3& x, D3& w) {
    int view, row, col;
    if (C.sensors) {
        view = (int)C.sensors[3 * px]; row = (int)C.sensors[3 * px + 1]; col = (int)C.sensors[3 * px + 2];
    } else {
        const long long hw = (long long)C.height * C.width;
        view = (int)(px / hw);
        const int rem = (int)(px - (long long)view * hw);
        row = rem / C.width;
        col = rem % C.width;
    }
    const float* p = C.poses + 9 * view;
    const D3 o = d3((double)p[0], (double)p[1], (double)p[2]), dd = d3((double)p[3], (double)p[4], (double)p[5]),
             n = d3((double)p[6], (double)p[7], (double)p[8]);
    double sx_ = 0.5, sy_ = 0.5;
    if (C.jittered) { sx_ = uni(rng); sy_ = uni(rng); }
    const double znear = (double)C.znear;
    const double sx = (((double)col + sx_) * 2.0 - (double)C.width) * znear / (double)C.height;
    const double sy = (((double)row + sy_) * 2.0 - (double)C.height) * znear / (double)C.height;
    const double sz = znear / tan((double)C.fov * 0.5);
    const D3 zaxis = normd(dd), xaxis = normd(crossd(n, zaxis)), yaxis = crossd(zaxis, xaxis);
    w = xaxis * sx + yaxis * sy + zaxis * sz;
    x = o + w;
    w = normd(w);
}

// include/vr_path_integrator_NEE.h:1-66 (+ directional light, bounce cap)
__device__ D3 path_nee_d(const DMedium& M, Rng& rng, D3 x, D3 w, uint32_t& verts, uint32_t* status) {
    double tMin, tMax;
    boundary_d(M, x, w, tMin, tMax);
    x = x + w * tMin;
    double d = tMax - tMin;
    const D3 env = d3(M.env);
    D3 R = env * transmittance_d(M, rng, x, w, status), W = d3(1.0, 1.0, 1.0);
    const double EPS = 0.00001;
    int bounces = 0;
    const D3 sun_dir = d3(M.sun_dir), sun_L = d3(M.sun_L);
    FlightD ff;
    for (int it = 0; d > EPS; ++it) {
        if (it >= (1 << 26)) {
            raise_status(status, 4);
            break;
        }
        double md;
        const double m = dmax(EPS, ff.bk.query(M, x, w, md));
        const double t = ff.sample(rng) / m;
        x = x + w * dmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.t += t;
        const double s = sigma_d(M, x);
        if (uni(rng) >= s / m) { d -= t; continue; }
        ++verts;
        const D3 sa = albedo_d(M, x);
        R = R + W * (d3(1.0, 1.0, 1.0) - sa) * d3(M.emission);
        W = W * sa;
        const D3 wnee = random_direction_d(rng, d3(0.0, 1.0, 0.0));
        const D3 Le = env * (4.0 * kPiD);
        const double Tn = transmittance_d(M, rng, x, wnee, status);
        R = R + W * Tn * Le * phase_d(M, w, wnee);
        if (M.has_sun) {
            const double Ts = transmittance_d(M, rng, x, sun_dir, status);
            R = R + W * Ts * sun_L * phase_d(M, w, sun_dir);
        }
        ++bounces;
        if (M.max_bounces > 0 && bounces >= M.max_bounces) break;
        const D3 wo = phase_sample_d(M, rng, w);
        if (W.x < EPS && W.y < EPS && W.z < EPS) break;
        w = wo;
        boundary_d(M, x, w, tMin, d);
        ff.bk.live = false;
    }
    return R;
}

__global__ void __launch_bounds__(128) k_capture_fp64(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                      double* __restrict__ out, double scale, DScratch* sc) {
    uint32_t verts = 0, paths = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n_paths; base += stride) {
        const uint64_t pid = base + threadIdx.x;
        if (pid >= n_paths) continue;
        Rng rng;
        rng.init(seed, pid, 0);
        const long long px = (long long)(pid % (uint64_t)S.npix);
        D3 x, w;
        camera_d(S.cam, px, rng, x, w);
        const D3 R = path_nee_d(M, rng, x, w, verts, &sc->status);
        atomicAdd(out + 3 * px + 0, R.x * scale);
        atomicAdd(out + 3 * px + 1, R.y * scale);
        atomicAdd(out + 3 * px + 2, R.z * scale);
        ++paths;
    }
    unsigned long long p = paths, v = verts;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p += __shfl_down_sync(0xffffffffu, p, o);
        v += __shfl_down_sync(0xffffffffu, v, o);
    }
    if ((threadIdx.x & 31u) == 0u) {
        if (p) atomicAdd(&sc->paths, p);
        if (v) atomicAdd(&sc->vertices, v);
    }
}

}  // namespace

int launch_capture_fp64(const DMedium& M, const PathSrc& S, int spp, uint64_t seed, double* rgb, DScratch* sc,
                        int num_sms, cudaStream_t stream) {
    const uint64_t n = (uint64_t)S.npix * (uint64_t)spp;
    if (n == 0) return VRT_OK;
    uint64_t blocks = (n + 127) / 128;
    const uint64_t cap = (uint64_t)num_sms * 32;
    if (blocks > cap) blocks = cap;
    k_capture_fp64<<<(int)blocks, 128, 0, stream>>>(M, S, n, seed, rgb, 1.0 / (double)spp, sc);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

}  // namespace vrt
