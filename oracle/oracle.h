/*
 * oracle.h -- CPU oracle for the volumetric path-integration hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * (rendervous_b200/csrc, exported through include/vrt.h) is compared against.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it; the product never links or calls it.
 *
 * It is a sequential restatement of the reference's GLSL (rendervous
 * include/ headers), one function per reference function, each citing the file and
 * lines it follows.  Two deliberate substitutions, applied identically on the
 * GPU side:
 *   - the hybrid Tausworthe RNG (include/randoms.h:6-59) is replaced by a
 *     counter-based Philox-4x32-10 keyed per path, so that any draw of any path
 *     can be regenerated without storing state;
 *   - the majorant map may be the reference's global constant
 *     (_objects.py:96-101) or a bricked majorant grid (an extension with no
 *     reference counterpart).
 *
 * PARITY UNPINNED: the reference ships no tests, golden vectors or fixtures
 * for this path, and its GLSL runs only under Vulkan (absent here), so this
 * restatement cannot be checked against reference outputs.  It is pinned
 * instead by analytic known-answer tests (homogeneous exp(-sigma d),
 * piecewise-constant DDA, closed-form trilinear segment integrals, HG moments,
 * finite differences) in tests/test_oracle_*.py.
 */
#ifndef VRT_ORACLE_H
#define VRT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
/* CDEF-BEGIN */
typedef struct orc_grid {
    const float* data;   /* contiguous [D,H,W,C] float32 */
    float* grad;         /* same layout, may be NULL */
    int32_t D, H, W, C;
} orc_grid;

typedef struct orc_scene {
    orc_grid sigma;               /* Grid3D sigma (C == 1) */
    float bmin[3], bmax[3];       /* Grid3D box */
    float inv_bsize[3];           /* 1/(bmax-bmin) computed in float32 by the host */
    float box_min[3], box_max[3]; /* boundary (RayBoxIntersection) box */
    int32_t albedo_is_grid;
    orc_grid albedo;              /* C == 1 or 3, same box as sigma */
    float albedo_const[3];
    float emission[3];
    float env[3];                 /* constant environment radiance */
    int32_t has_sun;
    float sun_dir[3];             /* unit direction towards the light */
    float sun_radiance[3];
    int32_t phase_mode;           /* 0 Henyey-Greenstein, 1 reference HGPhase+VHGPhaseSampler mixture */
    float phase_g;
    int32_t majorant_mode;        /* 0 global constant, 1 majorant grid */
    float global_majorant;
    const float* maj_grid;        /* [Mz,My,Mx] */
    int32_t maj_dims[3];          /* Mx, My, Mz */
    float maj_scale[3];           /* inv_bsize * dim / brick */
    int32_t transmittance_mode;   /* 0 RT, 1 DT, 2 DDA midpoint, 3 DDA exact, 4 GRT, 5 GDT */
    int32_t max_bounces;          /* 0 = uncapped (reference) */
    float ds_epsilon;
    int32_t ds_compat;            /* 1 = reference replay majorant quirk in NEE_DS bw */
    int32_t exitance_mode;        /* collision integrators: 0 emission, 1 scattered, 2 scattered + emitted */
    int32_t emission_is_grid;     /* emission: 0 const emission[3], 1 emission_grid (C 1 or 3, sigma's box) */
    orc_grid emission_grid;
    int32_t env_mode;             /* 0 constant env[3], 1 equirectangular image env_image [H, W, 3] */
    const float* env_image;
    int32_t env_hw[2];
    int32_t env_sampler;          /* NEE directions: 0 uniform sphere, 1 the image's quadtree */
    const float* env_quadtree;    /* 4 + 16 + ... + 4^env_levels node probabilities */
    int32_t env_levels;
} orc_scene;

typedef struct orc_camera {
    const float* poses;           /* [views, 9] origin, direction, up */
    int32_t views, height, width;
    float fov, znear;
    int32_t jittered;
    const int64_t* sensors;       /* NULL: every pixel; else [n_sensors, 3] (view, row, col) */
    int64_t n_sensors;
} orc_camera;

typedef struct orc_counters {
    int64_t paths, vertices, steps;
} orc_counters;

void orc_set_threads(int32_t n);
int32_t orc_get_threads(void);

void orc_philox4x32_10(uint32_t key0, uint32_t key1, const uint32_t ctr[4], uint32_t out[4]);
void orc_random_sequence(uint64_t seed, uint64_t path, uint32_t stream, uint32_t start, int32_t n, float* out);

void orc_ray_box(const float* rays, int64_t n, const float bmin[3], const float bmax[3], float* out2);
void orc_grid3d_fw(const orc_grid* g, const float bmin[3], const float inv_bsize[3], const float* x, int64_t n, float* out);
void orc_grid3d_bw(const orc_grid* g, const float bmin[3], const float inv_bsize[3], const float* x, const float* dout, int64_t n);

void orc_majorant_build(const orc_grid* sigma, int32_t brick, float* out, int32_t dims_out[3]);
void orc_majorant_query(const orc_scene* s, const float* rays, int64_t n, float* out2);

/* mode: 0 RT, 1 DT, 2 DDA midpoint, 3 DDA exact, 4 GRT, 5 GDT (forward only) */
void orc_transmittance_fw(const orc_scene* s, int32_t mode, const float* rays, int64_t n, uint64_t seed, int32_t fp64, float* T);
void orc_transmittance_bw(const orc_scene* s, int32_t mode, const float* rays, int64_t n, uint64_t seed, const float* dL_dT);
/* The DDA's optical depth (midpoint or exact rule) in FP64 */
void orc_dda_tau_fp64(const orc_scene* s, int32_t exact, const float* rays, int64_t n, double* tau);
/* FP64 fine ray-march of tau = int sigma along the ray, sigma read with the DDA-side clamping lookup */
void orc_tau_raymarch_fp64(const orc_scene* s, const float* rays, int64_t n, int32_t substeps, double* tau);

void orc_phase_sample(const orc_scene* s, const float* w_in, int64_t n, uint64_t seed, float* out4);
void orc_env_sample(const orc_scene* s, int64_t n, uint64_t seed, float* out6);

void orc_camera_rays(const orc_camera* cam, int32_t spp, uint64_t seed, float* out6);

/* integrator: 0 NEE (DS/DRT/... forward), 1 DT (no NEE), 2 MC collision integrator, 3 DDA collision integrator */
void orc_radiance_fw(const orc_scene* s, int32_t integrator, const float* rays, int64_t n, uint64_t seed, float* R, orc_counters* c);
/* bw_mode: 0 NEE_DS, 1 DT, 2 NEE_DRT, 3 DRTQ, 4 DRTDS, 5 SPS, 6 MC collision integrator, 7 DDA collision integrator */
/* DeltatrackingCollisionSampler on rays: out3 [n,3] = (C, t, T); bw scatters dL/d(C, T) */
void orc_collision_sample_fw(const orc_scene* s, const float* rays, int64_t n, uint64_t seed, float* out3);
void orc_collision_sample_bw(const orc_scene* s, const float* rays, int64_t n, uint64_t seed, const float* dL_dout3);
void orc_radiance_bw(const orc_scene* s, int32_t bw_mode, const float* rays, int64_t n, uint64_t seed, const float* dL_dR);

void orc_capture_fw(const orc_scene* s, int32_t integrator, const orc_camera* cam, int32_t spp, uint64_t seed, float* rgb, orc_counters* c);
void orc_capture_bw(const orc_scene* s, int32_t bw_mode, const orc_camera* cam, int32_t spp, uint64_t seed, const float* dL_drgb);
/* The NEE capture with every quantity in double: rgb [pixels, 3] doubles */
void orc_capture_fw_fp64(const orc_scene* s, const orc_camera* cam, int32_t spp, uint64_t seed, double* rgb);
/* Radiance-cache forms of the NEE capture.  prefix: paths stop at their
   (cut+1)-th real collision; rgb += prefix / spp; queries = 3 planes [n,3]
   (position, direction, throughput W; W = 0 where the path ended earlier),
   n = spp * pixels, row = Philox path id.  train: n_paths paths from pixels
   drawn by each path's first u32; samples = 4 planes [n_paths*rec, 3]
   (position, direction, target (R_final - R_k)/W_k, W_k); unused rows have
   NaN targets; rec <= 8.  cut >= 0 stops training paths at their (cut+1)-th
   collision with nothing added for the rest (a cache that returns 0). */
void orc_capture_prefix(const orc_scene* s, const orc_camera* cam, int32_t spp, uint64_t seed, int32_t cut, float* rgb,
                        float* queries);
void orc_train_samples(const orc_scene* s, const orc_camera* cam, int64_t n_paths, uint64_t seed, int32_t rec,
                       int32_t cut, float* samples);
/* CDEF-END */
#ifdef __cplusplus
}
#endif
#endif
