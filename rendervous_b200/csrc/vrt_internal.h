// vrt_internal.h -- host-side declarations shared by the libvrt translation units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "vrt_params.h"

struct vrt_context {
    int device;
    int num_sms;
    vrt::DScratch* scratch;  // device memory
    void* wave;              // wavefront job buffer (grown on demand)
    size_t wave_bytes;
    unsigned long long log_limit;  // NEE_DS collision-log cap in records (0: automatic)
    unsigned long long batch_limit;  // wavefront items per round beyond the reserve (0: automatic)
};

namespace vrt {

// Returns VRT_OK or VRT_E_CUDA after checking the launch.
int launch_status(cudaError_t e);

// Grows the context's wavefront buffer to at least `bytes` (contents undefined).
int ensure_wave_buffer(vrt_context* ctx, size_t bytes);

// Host-side count of the kernels this library launched (vrt_launch_count).
void count_launches(int n);

// Brackets one launch of wavefront kernel `kid` (VRT_K_*): counts it and, with
// kernel timing on, records CUDA events before and after it on `stream`.
struct KernelScope {
    int kid;
    cudaStream_t stream;
    cudaEvent_t e0, e1;
    KernelScope(int kid, cudaStream_t stream);
    ~KernelScope();
};

// Wavefront NEE_DS adjoint (vrt_wave.cu): capped paths, default replay majorant.
int launch_wave_ds_bw(vrt_context* ctx, const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                      const float* dL, float div, cudaStream_t stream);

// Wavefront NEE forward (vrt_wave.cu), capped paths only.
// cut >= 0: a path stops at its (cut+1)-th real collision and writes its
// radiance-cache query there (3 planes of `n_paths` rows in `queries`: position,
// arrival direction, throughput; zeros when it never gets there).
int launch_wave_fw(vrt_context* ctx, const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed, float* out,
                   float scale, cudaStream_t stream, int cut = -1, float* queries = nullptr);

int persistent_blocks(const void* kernel, int block, int num_sms);

// num_sms < 1: the DDA modes' persistent grid is sized from the device's SM count
int launch_transmittance_fw(const DMedium& M, int mode, const float* rays, int64_t n, uint64_t seed, float* T,
                            DScratch* scratch, int num_sms, cudaStream_t stream);
// tmp: n floats (the DDA modes' dL/dtau per ray between their two marches)
int launch_transmittance_bw(const DMedium& M, int mode, const float* rays, int64_t n, uint64_t seed,
                            const float* dL_dT, float* tmp, DScratch* scratch, int num_sms, cudaStream_t stream);

// out: rays mode writes R [n,3]; camera mode accumulates R * scale into out[pixel].
int launch_radiance_fw(const DMedium& M, int integrator, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                       float* out, float scale, DScratch* scratch, int num_sms, cudaStream_t stream);
// dL: rays mode dL[i]; camera mode dL[pixel] / div (div = spp, as the reference's
// capture backward divides dL/dI by the sample count, _maps.py:707-708).
// pids: the n_paths paths listed there (device array), else paths 0 .. n_paths-1.
int launch_radiance_bw(const DMedium& M, int bw_mode, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                       const float* dL, float div, DScratch* scratch, int num_sms, cudaStream_t stream,
                       const unsigned long long* pids = nullptr);

// Wavefront DRT / DRTDS adjoint (vrt_wave_drt.cu; bw_mode VRT_BW_NEE_DRT or
// VRT_BW_NEE_DRTDS): capped paths, ratio or delta tracking light rays; and its
// per-path reservoir branch (vrt_path.cu; ds: the DRTDS form) over the round's
// paths [p_begin, min(*next_path, n_paths)) (at most max_round).
int launch_wave_drt_bw(vrt_context* ctx, const DMedium& M, int bw_mode, const PathSrc& src, uint64_t n_paths,
                       uint64_t seed, const float* dL, float div, cudaStream_t stream);
// Wavefront SPS adjoint (vrt_wave_sps.cu): ratio or delta tracking light rays.
int launch_wave_sps_bw(vrt_context* ctx, const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                       const float* dL, float div, cudaStream_t stream);
// The DRT-family branches (vrt_path.cu): mode 0 DRT, 1 DRTDS (one per path of
// the round), 2 DRTQ (one scatter term per segment: segment 0s in resv, then
// *n_segs in segs).  items / post: 3 float4 per branch each, R: 3 floats each,
// n_items: 2 counters.
int launch_drt_branch(const DMedium& M, int mode, const PathSrc& src, uint64_t n_paths, uint64_t p_begin,
                      const unsigned long long* next_path, uint64_t seed, const float* dL, float div, const float* info,
                      const float4* resv, uint64_t max_round, const float4* segs, const unsigned long long* n_segs,
                      uint64_t max_segs, float4* items, float4* post, float* R, unsigned long long* n_items,
                      DScratch* scratch, int num_sms, cudaStream_t stream);

// Radiance-cache forms of the forward NEE kernel (mode FW_CUT or FW_TRAIN).
int launch_cache_paths(const DMedium& M, int mode, const PathSrc& src, uint64_t n_paths, uint64_t seed, float* out,
                       float scale, const CacheIO& io, DScratch* scratch, int num_sms, cudaStream_t stream);
// Training targets from the recorded collisions and the per-path estimates.
int launch_cache_targets(float* smp, const float* pR, long long n_paths, int rec, cudaStream_t stream);

// Collision integrators (vrt_collision.cu): integrator VRT_PI_MC_COLLISION or
// VRT_PI_DDA_COLLISION; out / dL as in launch_radiance_fw / _bw.
int launch_collision_fw(const DMedium& M, int integrator, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                        float* out, float scale, DScratch* scratch, int num_sms, cudaStream_t stream);
int launch_collision_bw(const DMedium& M, int integrator, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                        const float* dL, float div, DScratch* scratch, int num_sms, cudaStream_t stream);
// DeltatrackingCollisionSampler on rays: forward when out3 != null, else backward with dL3.
int launch_collision_sample(const DMedium& M, const float* rays, int64_t n, uint64_t seed, float* out3,
                            const float* dL3, DScratch* scratch, int num_sms, cudaStream_t stream);

// The FP64 NEE capture (vrt_fp64.cu): rgb [pixels, 3] doubles, accumulated.
int launch_capture_fp64(const DMedium& M, const PathSrc& S, int spp, uint64_t seed, double* rgb, DScratch* sc,
                        int num_sms, cudaStream_t stream);

// The NEE_DS adjoint as a persistent state machine (vrt_adjoint.cu); with
// pids, over the n_paths paths listed there (device array).
int launch_nee_ds_bw(const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed, const float* dL,
                     float div, DScratch* scratch, int num_sms, cudaStream_t stream,
                     const unsigned long long* pids = nullptr);

}  // namespace vrt
