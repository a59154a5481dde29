/*
 * vrt.h -- C ABI of libvrt.so, the B200 (sm_100a) volumetric path-integration
 * library.  This is the drop-in boundary for rendervous's volume hot path: the
 * Python map classes in rendervous_b200/ lower a map graph to the plain
 * structs below and call these entry points through cffi.
 *
 * Conventions
 *   - Every pointer argument that names tensor data is a DEVICE pointer of the
 *     current CUDA device; `stream` is a cudaStream_t (NULL = legacy stream).
 *   - Every call is asynchronous on `stream` and returns a status code
 *     (VRT_OK == 0).  Argument errors are reported before any launch; device
 *     side failures (an iteration cap hit, a non-finite value) are recorded in
 *     the context and returned by vrt_context_sync().
 *   - Gradient outputs ACCUMULATE into the grad buffers named in the structs
 *     (the reference binds and accumulates into `param.grad`,
 *     rendervous _maps.py:1049-1058); the library never zeroes them.
 *   - Random numbers: draw k of path p is word (k & 3) of
 *     Philox-4x32-10(key = seed, counter = {k >> 2, p_lo, stream, p_hi}), so a
 *     call with the same seed regenerates the same paths.
 *   - A context serialises nothing: use one context per stream.
 */
#ifndef VRT_H
#define VRT_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
/* CDEF-BEGIN */
enum {
    VRT_OK = 0,
    VRT_E_INVALID_ARGUMENT = 1,
    VRT_E_NULL_POINTER = 2,
    VRT_E_BAD_SHAPE = 3,
    VRT_E_ITER_CAP = 4,
    VRT_E_NONFINITE = 5,
    VRT_E_CUDA = 6,
    VRT_E_UNSUPPORTED = 7
};

/* Transmittance estimators (the transmittance sub-maps of the reference). */
enum {
    VRT_TR_RATIO_TRACKING = 0,  /* RatiotrackingTransmittance, include/vr_transmittance_RT.h */
    VRT_TR_DELTA_TRACKING = 1,  /* DeltatrackingTransmittance, include/vr_transmittance_DT.h */
    VRT_TR_DDA_MIDPOINT = 2,    /* GridDDATransmittance, include/vr_transmittance_DDA.h */
    VRT_TR_DDA_EXACT = 3,       /* DDA with the exact per-cell trilinear integral (no reference) */
    VRT_TR_GRID_RATIO = 4,      /* GridRatiotrackingTransmittance, include/vr_transmittance_GRT.h (forward only) */
    VRT_TR_GRID_DELTA = 5       /* GridDeltatrackingTransmittance, include/vr_transmittance_GDT.h (forward only) */
};
/* Integrator forward passes: the path integrators, and the collision
   integrators MCCollisionIntegrator (include/maps/collision_integrator_mc.h)
   and GridDDACollisionIntegrator (include/vr_collision_integrator_DDA.h),
   whose exitance radiance is vrt_medium.exitance_mode. */
enum { VRT_PI_NEE = 0, VRT_PI_DT = 1, VRT_PI_MC_COLLISION = 2, VRT_PI_DDA_COLLISION = 3 };
/* Path-replay adjoints (DeltatrackingNEEPathIntegrator, DeltatrackingPathIntegrator,
   DRTPathIntegrator, DRTQPathIntegrator, DRTDSPathIntegrator, SPSPathIntegrator;
   include/vr_path_integrator_NEE_DS.h, _DT.h, _NEE_DRT.h, _NEE_DRTQ.h, _NEE_DRTDS.h, _NEE_SPS.h). */
enum {
    VRT_BW_NEE_DS = 0,
    VRT_BW_DT = 1,
    VRT_BW_NEE_DRT = 2,
    VRT_BW_NEE_DRTQ = 3,
    VRT_BW_NEE_DRTDS = 4,
    VRT_BW_NEE_SPS = 5,
    VRT_BW_MC_COLLISION = 6,    /* MCCollisionIntegrator BACKWARD (collision_integrator_mc.h:20-41) */
    VRT_BW_DDA_COLLISION = 7    /* GridDDACollisionIntegrator BACKWARD (vr_collision_integrator_DDA.h:85-207) */
};

/* A node-centred FP32 grid, the Grid3D parameter (rendervous _maps.py:2319-2365).
   Element (z,y,x,c) is data[z*strides[0] + y*strides[1] + x*strides[2] + c]; with
   C > 1 the channel stride must be 1.  grad uses the same strides and may be NULL. */
typedef struct vrt_grid {
    const float* data;
    float* grad;
    int32_t shape[4];    /* D, H, W, C */
    int64_t strides[4];  /* element strides of D, H, W, C */
} vrt_grid;

/* A lowered medium: the sub-maps a path integrator binds
   (rendervous _maps.py:2924-3022) reduced to the forms this library runs. */
typedef struct vrt_medium {
    vrt_grid sigma;                  /* Grid3D, C == 1 */
    float bmin[3], bmax[3];          /* Grid3D box */
    float inv_bsize[3];              /* 1/(bmax-bmin), float32 */
    float box_min[3], box_max[3];    /* RayBoxIntersection boundary */
    int32_t albedo_is_grid;          /* 0: albedo_const, 1: albedo grid (C 1 or 3, Grid3D box) */
    vrt_grid albedo;
    float albedo_const[3];
    float emission[3];               /* constant emission */
    float env[3];                    /* constant environment radiance */
    int32_t has_sun;                 /* directional light (no reference counterpart) */
    float sun_dir[3];                /* unit direction towards the light */
    float sun_radiance[3];
    int32_t phase_mode;              /* 0 Henyey-Greenstein, 1 HGPhase + VHGPhaseSampler (reference) */
    float phase_g;
    int32_t majorant_mode;           /* 0 constant [max, 1e6] (reference), 1 majorant grid */
    float global_majorant;
    const float* maj_grid;           /* [Mz, My, Mx] from vrt_majorant_build */
    int32_t maj_dims[3];             /* Mx, My, Mz */
    float maj_scale[3];              /* inv_bsize * (shape-1) / brick */
    int32_t transmittance_mode;      /* VRT_TR_* used for NEE shadow rays */
    int32_t max_bounces;             /* 0 = uncapped, as the reference */
    float ds_epsilon;                /* defensive-sampling epsilon of the DS / DT adjoints and the collision sampler */
    int32_t ds_compat;               /* 1: reference replay majorant of NEE_DS bw */
    /* exitance radiance of the collision integrators (VRT_PI_MC_COLLISION, VRT_PI_DDA_COLLISION):
       0 the emission (ds.exitance_radiance = ds.emission), 1 MCScatteredRadiance,
       2 MCScatteredEmittedRadiance (_maps.py:2730-2760; radiance = transmittance x environment) */
    int32_t exitance_mode;
    int32_t emission_is_grid;        /* 0: emission[3] constant; 1: emission_grid (Grid3D, C 1 or 3, sigma's box) */
    vrt_grid emission_grid;
    /* environment (_objects.py:165-199): 0 the constant env[3]; 1 an equirectangular
       image env_image [env_hw[0], env_hw[1], 3] (Image2D(img).after(xr_projection)),
       not differentiated.  NEE directions: env_sampler 0 uniform sphere
       (UniformDirectionSampler), 1 the image's probability quadtree
       (XRQuadtreeRandomDirection; env_quadtree holds 4 + 16 + ... + 4^env_levels
       node probabilities, children of node k at 4k+1..4k+4 in Morton order). */
    int32_t env_mode;
    const float* env_image;
    int32_t env_hw[2];
    int32_t env_sampler;
    const float* env_quadtree;
    int32_t env_levels;
} vrt_medium;

/* PerspectiveCameraSensor (rendervous _maps.py:1765-1802).  sensors == NULL:
   every pixel of every view (image [views, H, W, 3]); else a sensors batch of
   n_sensors (view, row, col) triples (SensorsBase.capture's sensors_batch,
   _maps.py:1741-1749; image [n_sensors, 3], sample s of sensor k is Philox
   path id s * n_sensors + k).  A triple outside the camera is recorded as
   VRT_E_INVALID_ARGUMENT (returned by vrt_context_sync) and its pixel's value
   is undefined. */
typedef struct vrt_camera {
    const float* poses;              /* [views, 9]: origin, direction, up */
    int32_t views, height, width;
    float fov, znear;
    int32_t jittered;
    const int64_t* sensors;          /* device [n_sensors, 3] int64, or NULL */
    int64_t n_sensors;
} vrt_camera;

typedef struct vrt_counters {
    int64_t paths;                   /* paths started */
    int64_t vertices;                /* real scattering collisions */
    int64_t steps;                   /* tracking steps (free-flight samples, DDA cells), primary and shadow */
    int64_t lookups;                 /* sigma lookups (8 node gathers each; DDA: cells) */
    int64_t reds;                    /* gradient atomic adds issued */
    int64_t albedo_lookups;          /* albedo grid lookups */
    int64_t status;                  /* device error bits (VRT_E_* as 1 << code) */
    int64_t detail;                  /* which device guard raised it (bit per site; diagnostics) */
} vrt_counters;

typedef struct vrt_context vrt_context;

/* Context: device scratch for work queues, counters and the error word
   (replaces the reference's global pipeline caches, _maps.py:35-66). */
int vrt_context_create(int32_t device, vrt_context** out);
int vrt_context_destroy(vrt_context* ctx);
/* Waits for `stream`, copies the counters and error word out, and clears them.
   Returns VRT_OK or the first device-side error. */
int vrt_context_sync(vrt_context* ctx, void* stream, vrt_counters* out);
const char* vrt_status_string(int32_t status);
/* Number of kernels this library has launched in the process (for launch accounting). */
int64_t vrt_launch_count(void);

/* Per-kernel measurement of the wavefront kernels (no reference counterpart).
   Each kernel adds its own tallies (tracking steps, sigma lookups, atomic adds,
   albedo lookups, bytes of the NEE_DS collision log written or read) to a slot
   of the context; with timing on, the library also brackets every launch with
   CUDA events on its stream.  vrt_kernel_stats waits for `stream`, fills
   VRT_K_COUNT entries (launches, event time summed in ms, tallies) accumulated
   since its last call, and clears them.  The replay's `steps` are the logged
   collisions it replayed. */
enum {
    VRT_K_WALK_FW = 0,     /* forward walk (primary paths, shadow jobs) */
    VRT_K_SHADOW_FW = 1,   /* forward shadow transmittances */
    VRT_K_DS_PRIMAL = 2,   /* NEE_DS adjoint: primal walk (writes the collision log) */
    VRT_K_SHADOW_T = 3,    /* NEE_DS (DRT, DRTDS, SPS) adjoint: the primal's light-ray transmittances */
    VRT_K_DS_REPLAY = 4,   /* NEE_DS adjoint: replay of the logged collisions (sigma / albedo scatters) */
    VRT_K_SHADOW_ADJ = 5,  /* NEE_DS (DRT, DRTDS, SPS) adjoint: the light rays' transmittance adjoints */
    VRT_K_DS_REWALK = 6,   /* NEE_DS adjoint: replay walk of the paths the log could not hold */
    VRT_K_DRT_PRIMAL = 7,  /* DRT adjoint: primal walk (collision log, light jobs, reservoir) */
    VRT_K_DRT_REPLAY = 8,  /* DRT adjoint: replay of the logged collisions (sigma scatters) */
    VRT_K_DRT_BRANCH = 9,  /* DRT adjoint: the reservoir vertex's branch, one per path */
    VRT_K_SPS_PRIMAL = 10, /* SPS adjoint: primal walk (segment log, light jobs) */
    VRT_K_SPS_REPLAY = 11, /* SPS adjoint: replay of the logged vertices (sigma and dL/dtau scatters) */
    VRT_K_COUNT = 12
};
typedef struct vrt_kernel_stat {
    int64_t launches;
    double ms;                       /* 0 unless timing was on */
    int64_t steps, lookups, reds, albedo_lookups, log_bytes;
} vrt_kernel_stat;
/* Caps the NEE_DS collision log of a context at `events` collision records
   (32 bytes each) per round; 0 restores the automatic size.  Paths whose
   collisions do not fit are replayed by walking them again (same gradients,
   more time). */
int vrt_set_collision_log_limit(vrt_context* ctx, int64_t events);
/* Caps the items (shadow jobs, vertex records) a wavefront round holds beyond
   the worst case of the paths in flight; 0 restores the automatic size (up to
   2^27).  A smaller cap means a smaller device footprint and more rounds;
   uncapped paths that outgrow a round's room resume in the next round
   (forward) or finish on the state-machine adjoint (NEE_DS); results are the
   same up to the order of float sums. */
int vrt_set_wave_batch_limit(vrt_context* ctx, int64_t items);
void vrt_set_kernel_timing(int32_t on);
/* Gather microbenchmark (the roofline of the lookups): threads x per_thread
   random 32-byte loads (L1 bypassed) from `buffer` (bytes long, 32-byte
   aligned); the caller times it.  sink: one device uint32 the kernel may write. */
int vrt_gather_peak(const void* buffer, int64_t bytes, int64_t threads, int32_t per_thread, uint32_t seed,
                    uint32_t* sink, void* stream);
/* Atomic-add microbenchmark (the roofline of the gradient scatters): threads x
   per_thread float atomic adds of 1/2^20 at random words of `buffer` (n floats,
   4-byte aligned); pairs != 0 adds x-neighbour pairs with one vector atomic
   (two adds each).  The caller times it; buffer's contents change. */
int vrt_atomic_peak(float* buffer, int64_t n, int64_t threads, int32_t per_thread, int32_t pairs, uint32_t seed,
                    void* stream);
int vrt_kernel_stats(vrt_context* ctx, void* stream, vrt_kernel_stat* out);
int32_t vrt_version(void);

/* RayBoxIntersection forward (rendervous _maps.py:4128-4154, include/maths.h:28-38):
   rays [n,6] -> out [n,2] = (tMin, tMax). */
int vrt_ray_box(const float* rays, int64_t n, const float bmin[3], const float bmax[3], float* out, void* stream);

/* Grid3D forward / backward (include/maps/grid3d.h:6-75): x [n,3] -> out [n,C];
   backward accumulates dL/dgrid into g->grad. */
int vrt_grid3d_fw(const vrt_grid* g, const float bmin[3], const float inv_bsize[3], const float* x, int64_t n,
                  float* out, void* stream);
int vrt_grid3d_bw(const vrt_grid* g, const float bmin[3], const float inv_bsize[3], const float* x,
                  const float* dout, int64_t n, void* stream);

/* Majorant grid of brick^3-cell bricks over sigma (the reference's only majorant
   is the constant of _objects.py:96-101).  With out == NULL only dims_out
   (Mx, My, Mz) is written. */
int vrt_majorant_build(const vrt_grid* sigma, int32_t brick, float* out, int32_t dims_out[3], void* stream);

/* Transmittance map forward / backward on rays [n,6] -> T [n]
   (GridDDATransmittance _maps.py:2640-2667, RatiotrackingTransmittance
   _maps.py:2670-2682, DeltatrackingTransmittance _maps.py:2685-2697).
   Backward accumulates dL/dsigma into medium->sigma.grad. */
int vrt_transmittance_fw(vrt_context* ctx, const vrt_medium* m, int32_t mode, const float* rays, int64_t n,
                         uint64_t seed, float* T, void* stream);
int vrt_transmittance_bw(vrt_context* ctx, const vrt_medium* m, int32_t mode, const float* rays, int64_t n,
                         uint64_t seed, const float* dL_dT, void* stream);

/* Transmittance forward for callers that cannot allocate device memory (no
   counterpart in the reference): code running inside another framework's
   pre-sized memory pool, or plugins that must not grow the device footprint.
   Same result as vrt_transmittance_fw, but it needs no vrt_context: with
   brick > 0 and a tracking mode (RT, DT) it builds the brick^3 majorant grid
   of m->sigma into a fixed array inside libvrt.so and tracks against it; with
   brick == 0 it uses m's own majorant.  The array holds at most 64^3 bricks
   (1 MiB, kept on every device that loads the library until exit); larger
   grids return VRT_E_BAD_SHAPE.  All calls share the array, so calls that
   overlap on the GPU race.  The first call in a CUDA context looks up the
   array's address; make it before any stream capture.  Every argument is
   checked before the first launch.  status_out == NULL: the call stays
   asynchronous and device-side errors (an iteration cap hit) are not
   reported.  status_out != NULL: the call waits for `stream`, stores the
   device error bits (1 << VRT_E_*) there and returns the first of them. */
int vrt_transmittance_fw_noalloc(const vrt_medium* m, int32_t mode, int32_t brick, const float* rays, int64_t n,
                                 uint64_t seed, float* T, int64_t* status_out, void* stream);

/* DeltatrackingCollisionSampler as a map on rays [n,6] -> out [n,3] = (C, t, T)
   (include/maps/collision_sampler_dt.h, _maps.py:2714-2727; ray i draws from
   stream 2 of Philox path i).  Backward takes dL/d(C, t, T) [n,3] (dL/dt is not
   propagated, as in the reference) and accumulates dL/dsigma into
   medium->sigma.grad from the defensively sampled walk (ds_epsilon). */
int vrt_collision_sample_fw(vrt_context* ctx, const vrt_medium* m, const float* rays, int64_t n, uint64_t seed,
                            float* out, void* stream);
int vrt_collision_sample_bw(vrt_context* ctx, const vrt_medium* m, const float* rays, int64_t n, uint64_t seed,
                            const float* dL_dout, void* stream);

/* Path integrator as a map on rays [n,6] -> R [n,3] (DeltatrackingPathIntegrator,
   DeltatrackingNEEPathIntegrator, DRTPathIntegrator, _maps.py:2886-3022; path i
   uses Philox path id i).  Backward accumulates into sigma.grad and albedo.grad. */
int vrt_radiance_fw(vrt_context* ctx, const vrt_medium* m, int32_t integrator, const float* rays, int64_t n,
                    uint64_t seed, float* R, void* stream);
int vrt_radiance_bw(vrt_context* ctx, const vrt_medium* m, int32_t bw_mode, const float* rays, int64_t n,
                    uint64_t seed, const float* dL_dR, void* stream);

/* Radiance cache (no reference counterpart): a 16-level dense grid encoding
   (2 features per level, FP32 parameters) plus degree-3 real spherical
   harmonics of the direction feed an MLP 64 -> 4 x 64 (ReLU) -> 16 (RGB in
   the first 3), run on the tensor cores with BF16 operands and FP32
   accumulation.  weights: W1..W4 [64][64] then W5 [16][64], row-major FP32.
   Level l of the grid is a (res[l]+1)^3 x 2 node array at the running offset
   of the previous levels; positions map to the grid through [bmin, bmax]. */
typedef struct vrt_cache {
    float* grid;
    float* grid_grad;
    float* weights;
    float* weights_grad;
    int32_t levels;                  /* must be 16 */
    int32_t res[16];
    float bmin[3], bmax[3];
} vrt_cache;
int64_t vrt_cache_grid_size(const int32_t res[16]);
/* MLP alone on given inputs [n,64] -> out [n,16] (tensor cores). */
int vrt_cache_mlp_fw(const float* weights, const float* inputs, int64_t n, float* out, void* stream);
/* Encoding + MLP: pos [n,3], dir [n,3] -> rgb [n,3]. */
int vrt_cache_infer(const vrt_cache* c, const float* pos, const float* dir, int64_t n, float* rgb, void* stream);
/* One pass of the relative-L2 loss sum_c (y_c - t_c)^2 / (y_c^2 + 0.01) (y held
   constant in the denominator) against target [n,3]; adds the sum over rows / n
   into *loss and accumulates the gradients into grid_grad and weights_grad.
   Rows with a non-finite target are skipped. */
int vrt_cache_train(const vrt_cache* c, const float* pos, const float* dir, const float* target, int64_t n,
                    float* loss, void* stream);
/* Adam step over n parameters (bias-corrected, step >= 1); clears grads. */
int vrt_cache_adam(float* params, float* grads, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                   float eps, int32_t step, void* stream);
/* Adds the cache's estimate for path-prefix queries (the planes written by
   vrt_capture_prefix_fw): rgb[row % npix] += scale * W[row] * cache(pos, dir). */
int vrt_cache_resolve(const vrt_cache* c, const float* queries, int64_t n, int64_t npix, float scale, float* rgb,
                      void* stream);
/* Waits for `stream`; returns VRT_OK, or VRT_E_ITER_CAP when a cache kernel
   gave up waiting for the tensor cores since the last call (and clears it). */
int vrt_cache_status(void* stream);

/* Camera capture (SensorsBase.capture, _maps.py:1741-1749, capture kernels
   _maps.py:509-746): rgb [views,H,W,3] = mean over spp paths; sample s of pixel p
   is Philox path id s*npix + p.  Backward replays the same paths with
   dL/drgb / spp and accumulates into the medium's grad buffers. */
int vrt_capture_fw(vrt_context* ctx, const vrt_medium* m, int32_t integrator, const vrt_camera* cam, int32_t spp,
                   uint64_t seed, float* rgb, void* stream);
int vrt_capture_bw(vrt_context* ctx, const vrt_medium* m, int32_t bw_mode, const vrt_camera* cam, int32_t spp,
                   uint64_t seed, const float* dL_drgb, void* stream);
/* The NEE capture in FP64 (no reference counterpart: the reference renders in
   FP32): the high-accuracy estimate that the radiance cache's error is
   measured against.  Same paths as vrt_capture_fw with VRT_PI_NEE (sample s
   of pixel p is Philox path s * npix + p), every quantity in double; rgb is a
   double [pixels, 3] (cleared here).  Supports constant environments with
   uniform NEE, ratio- or delta-tracking shadow rays, const or grid albedo and
   majorant; other media return VRT_E_UNSUPPORTED. */
int vrt_capture_fw_fp64(vrt_context* ctx, const vrt_medium* m, const vrt_camera* cam, int32_t spp, uint64_t seed,
                        double* rgb, void* stream);

/* Radiance-cache forms of the NEE capture (no reference counterpart).
   Prefix: the integrator of vrt_capture_fw, but a path stops at its (cut+1)-th
   real collision and records a query there; rgb ACCUMULATES prefix / spp (not
   cleared) and queries is 3 planes [n,3] (position, arrival direction,
   throughput; 0 throughput where the path ended before the cut), n = spp *
   pixels, row = Philox path id.  vrt_cache_resolve then adds the cache's part.
   Training samples: n_paths paths from pixels drawn by each path's first draw;
   with c == NULL they run to the end (the medium's bounce cap applies), else
   they stop into the cache c at their (cut+1)-th collision (cut >= rec), as
   the rendered paths do at theirs.  The first rec <= 8 collisions of path i
   fill rows i*rec.. of samples = 4 planes [n_paths*rec, 3]: position, arrival
   direction, in-scattered radiance target (R_final - R_k) / W_k and W_k.
   Rows of collisions the path never reached hold NaN targets, which
   vrt_cache_train skips.  work: 12 * n_paths floats of device scratch. */
int vrt_capture_prefix_fw(vrt_context* ctx, const vrt_medium* m, const vrt_camera* cam, int32_t spp, uint64_t seed,
                          int32_t cut, float* rgb, float* queries, void* stream);
int vrt_capture_train_samples(vrt_context* ctx, const vrt_medium* m, const vrt_camera* cam, const vrt_cache* c,
                              int32_t cut, int64_t n_paths, uint64_t seed, int32_t rec, float* samples, float* work,
                              void* stream);
/* CDEF-END */

#ifdef __cplusplus
}
#endif
#endif
