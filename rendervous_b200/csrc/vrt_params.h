// vrt_params.h -- kernel-parameter forms of the C-ABI structs.
//
// The host validates a vrt_medium / vrt_camera once per call and converts it
// to these POD structs, which are passed by value (they live in the kernel's
// constant bank, so every lane reads them as uniform values).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vrt {

struct DGrid {
    const float* data;
    float* grad;
    int D, H, W, C;
    int sD, sH, sW;  // element strides (channel stride is 1)
};

struct DMedium {
    DGrid sigma;
    DGrid albedo;
    float3 bmin, bmax, inv_bsize;
    float3 box_min, box_max;
    int albedo_is_grid;
    float3 albedo_const, emission, env;
    int has_sun;
    float3 sun_dir, sun_L;
    int phase_mode;
    float g;
    int maj_mode;
    float gmaj;
    const float* maj;
    int Mx, My, Mz;
    float3 maj_scale;
    int tr_mode;
    int max_bounces;
    float ds_eps;
    int ds_compat;
    int exitance_mode;     // collision integrators: 0 emission, 1 scattered, 2 scattered + emitted
    int emission_is_grid;  // emission: 0 const, 1 emission_grid
    DGrid emission_grid;
    int env_mode;          // environment: 0 the constant env, 1 an equirectangular (xr) image
    const float* env_img;  // [env_h, env_w, 3], contiguous
    int env_h, env_w;
    int env_sampler;       // NEE direction sampling: 0 uniform sphere, 1 the image's quadtree
    const float* env_qt;   // quadtree node probabilities (4 + 16 + ... + 4^levels floats)
    int env_levels;
};

struct DCamera {
    const float* poses;
    int views, height, width;
    float fov, znear;
    int jittered;
    const long long* sensors;  // [npix, 3] (view, row, col) of a sensors batch, or null: every pixel
};

// Device scratch owned by a context.
struct DScratch {
    unsigned long long next_path;  // persistent-kernel work queue
    unsigned long long paths;
    unsigned long long vertices;
    unsigned long long steps;
    unsigned long long lookups;
    unsigned long long reds;
    unsigned long long albedo;
    unsigned int status;           // 1 << VRT_E_* bits
    unsigned int detail;           // which guard raised a device error (bit per site)
    // per-kernel tallies of the wavefront kernels (VRT_K_*): steps, lookups, atomics, albedo lookups,
    // collision-log bytes; not cleared by vrt_context_sync, read and cleared by vrt_kernel_stats
    unsigned long long kstat[12][5];
};

}  // namespace vrt

namespace vrt {

// Source of primary rays for the path kernels: a camera (capture) or an array
// of rays [n, 6] (a path integrator evaluated as a map).
struct PathSrc {
    int is_camera;
    DCamera cam;
    long long npix;        // views * height * width (camera)
    const float* rays;     // [n, 6] (rays)
};

// Radiance-cache forms of the forward NEE kernel.
enum : int { FW_PLAIN = 0, FW_CUT = 1, FW_TRAIN = 2, FW_BRANCH = 3 };
struct CacheIO {
    int cut;         // >= 0: a path stops at its (cut+1)-th real collision and records a query there
                     // (always in FW_CUT; FW_TRAIN with cut < 0 traces full paths)
    int rec;         // FW_TRAIN: collisions recorded per path as training samples
    float* q;        // 3 planes [n_paths, 3]: position, direction, throughput (0: no query)
    float* smp;      // FW_TRAIN: 4 planes [n_paths*rec, 3]: position, direction, R at arrival, throughput
    float* pR;       // FW_TRAIN: [n_paths, 3] the path's estimate without its cache query; FW_BRANCH: the estimates
    long long rows;  // rows of a query plane (n_paths)
    // FW_BRANCH: per item 3 float4 -- start point and stream draw count, direction and fork count,
    // path id (low, high words) -- a scattered-only NEE path from a given stream position
    const float4* branch;
    unsigned long long* queue;  // FW_BRANCH: the items' work counter (zeroed by the caller)
};

}  // namespace vrt
