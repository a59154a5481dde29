// vrt_cache.cu -- the radiance cache: dense multiresolution grid encoding and a
// 64-wide MLP on the tcgen05 tensor cores (sm_100a).  No reference counterpart.
//
// Network: input 64 = 16 levels x 2 grid features + 16 real SH coefficients of
// the direction (degree 4) + a constant 1 (the first layer's bias) + zeros;
// four hidden layers of 64 with ReLU; 16 outputs of which 3 (RGB) are used.
// Weights are kept in FP32 (the optimiser's copy) and rounded to BF16 when a
// CTA stages them; products accumulate in FP32 in tensor memory.
//
// One CTA owns 128 samples: sample t of the tile is row t of every GEMM, lane
// t of TMEM, and thread t of the CTA.  Each layer is D[128 x N] = A[128 x K]
// B[N x K]^T issued by one thread as K/16 tcgen05.mma (kind::f16, BF16 inputs,
// FP32 accumulate) from BF16 tiles in shared memory, then read back per thread
// with tcgen05.ld.32x32b.  Tiles use the no-swizzle K-major core-matrix layout
// (8 rows x 16 bytes per 128-byte core matrix; LBO = next core matrix along K,
// SBO = next along M/N).  The backward pass multiplies by the transposed
// weights (staged separately) on the tensor cores; the weight gradients are
// 128-sample outer products on the CUDA cores.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/vrt.h"
#include "vrt_device.cuh"
#include "vrt_internal.h"

namespace vrt {
namespace cache {

constexpr int kTile = 128;
constexpr int kHid = 64, kOut = 16, kLevels = 16;
constexpr int kWaitIters = 1 << 22;

struct Enc {
    const float* grid;
    float* grid_grad;
    int res[kLevels];
    int off[kLevels];
    float3 bmin, inv_size;
};

// ------------------------------------------------------------- tile layout --
__device__ __forceinline__ uint32_t core_off(int r, int k, int K) {  // bytes, BF16 element (r, k)
    return (uint32_t)(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
// 8 consecutive values of row r starting at column k0 (k0 % 8 == 0) as one 16-byte store
__device__ __forceinline__ void store8(unsigned char* tile, int r, int k0, int K, const float* v) {
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 c = __floats2bfloat162_rn(v[4], v[5]), d = __floats2bfloat162_rn(v[6], v[7]);
    uint4 u;
    u.x = *reinterpret_cast<uint32_t*>(&a); u.y = *reinterpret_cast<uint32_t*>(&b);
    u.z = *reinterpret_cast<uint32_t*>(&c); u.w = *reinterpret_cast<uint32_t*>(&d);
    *reinterpret_cast<uint4*>(tile + core_off(r, k0, K)) = u;
}
__device__ __forceinline__ void load8(const unsigned char* tile, int r, int k0, int K, float* v) {
    uint4 u = *reinterpret_cast<const uint4*>(tile + core_off(r, k0, K));
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float2 f = __bfloat1622float2(h[i]);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// dynamic shared memory rounded up to 128 bytes (the launch adds 128 bytes of slack)
__device__ __forceinline__ unsigned char* smem_align128(unsigned char* p) {
    return p + ((128u - (smem_u32(p) & 127u)) & 127u);
}

// error word of the cache kernels (a tensor-core wait that ran out); read and
// cleared by vrt_cache_status
__device__ uint32_t g_cache_status;

// UMMA shared-memory descriptor, no swizzle, version 1 (sm100)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (int i = 0; i < kWaitIters; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Per-CTA GEMM engine: TMEM accumulator of 64 columns, one mbarrier.
struct Engine {
    uint32_t tmem, bar, phase;
    bool ok;

    // D[128 x n] = A[128 x k] * B[n x k]^T; A, B BF16 tiles in the core layout
    __device__ __forceinline__ void gemm(const unsigned char* A, const unsigned char* B, int n, int k) {
        // callers: every thread wrote its part of A (fence.proxy.async done) and synced
        if (threadIdx.x == 0) {
            fence_after();
            const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
            const uint32_t sbo = (uint32_t)(k >> 3) * 128u;
            for (int s = 0; s < k / 16; ++s)
                umma(tmem, sdesc(a0 + 256u * s, 128u, sbo), sdesc(b0 + 256u * s, 128u, sbo), idesc_bf16(n), s > 0 ? 1u : 0u);
            umma_commit(bar);
        }
    }
    // wait for the last gemm and read this thread's row (n columns, n % 16 == 0)
    __device__ __forceinline__ void read_row(int n, float* out) {
        bool done = mbar_wait(bar, phase);
        phase ^= 1u;
        if (!done) ok = false;
        fence_after();
        const uint32_t lane_base = (uint32_t)(threadIdx.x & ~31u) << 16;
        for (int c = 0; c < n; c += 16) tmem_ld16(tmem + lane_base + (uint32_t)c, out + c);
        tmem_wait_ld();
        fence_before();
    }
};

// ---------------------------------------------------------------- encoding --
__device__ __forceinline__ void sh4(float3 d, float* o) {
    // real spherical harmonics up to degree 3 (16 coefficients) with the
    // standard orthonormal constants
    const float x = d.x, y = d.y, z = d.z, xx = x * x, yy = y * y, zz = z * z;
    o[0] = 0.28209479177387814f;
    o[1] = -0.4886025119029199f * y;
    o[2] = 0.4886025119029199f * z;
    o[3] = -0.4886025119029199f * x;
    o[4] = 1.0925484305920792f * x * y;
    o[5] = -1.0925484305920792f * y * z;
    o[6] = 0.31539156525252005f * (2.0f * zz - xx - yy);
    o[7] = -1.0925484305920792f * x * z;
    o[8] = 0.5462742152960396f * (xx - yy);
    o[9] = -0.5900435899266435f * y * (3.0f * xx - yy);
    o[10] = 2.890611442640554f * x * y * z;
    o[11] = -0.4570457994644658f * y * (4.0f * zz - xx - yy);
    o[12] = 0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    o[13] = -0.4570457994644658f * x * (4.0f * zz - xx - yy);
    o[14] = 1.445305721320277f * z * (xx - yy);
    o[15] = -0.5900435899266435f * x * (xx - 3.0f * yy);
}

struct Corner8 {
    int idx[8];
    float wt[8];
};
__device__ __forceinline__ void level_corners(const Enc& E, int l, float3 u, Corner8& c) {
    const int R = E.res[l];
    const int R1 = R + 1;
    float gx = u.x * (float)R, gy = u.y * (float)R, gz = u.z * (float)R;
    int ix = min((int)gx, R - 1), iy = min((int)gy, R - 1), iz = min((int)gz, R - 1);
    float ax = gx - (float)ix, ay = gy - (float)iy, az = gz - (float)iz;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
        c.idx[k] = E.off[l] + (((iz + dz) * R1 + (iy + dy)) * R1 + (ix + dx)) * 2;
        c.wt[k] = (dx ? ax : 1.0f - ax) * (dy ? ay : 1.0f - ay) * (dz ? az : 1.0f - az);
    }
}
__device__ __forceinline__ float3 unit_coords(const Enc& E, float3 p) {
    float3 u = (p - E.bmin) * E.inv_size;
    u.x = fminf(fmaxf(u.x, 0.0f), 1.0f);
    u.y = fminf(fmaxf(u.y, 0.0f), 1.0f);
    u.z = fminf(fmaxf(u.z, 0.0f), 1.0f);
    return u;
}
// the 64 network inputs of one sample
__device__ __forceinline__ void encode(const Enc& E, float3 p, float3 d, float* x) {
    float3 u = unit_coords(E, p);
    for (int l = 0; l < kLevels; ++l) {
        Corner8 c;
        level_corners(E, l, u, c);
        float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float2 g = __ldg(reinterpret_cast<const float2*>(E.grid + c.idx[k]));
            f0 += c.wt[k] * g.x;
            f1 += c.wt[k] * g.y;
        }
        x[2 * l] = f0;
        x[2 * l + 1] = f1;
    }
    sh4(d, x + 32);
    x[48] = 1.0f;
#pragma unroll
    for (int i = 49; i < 64; ++i) x[i] = 0.0f;
}

// -------------------------------------------------------------- staging --
// Stage the FP32 weights as BF16 tiles: B operands W_l [n x k] and, when
// `transposed`, W_l^T [k x n] for the backward pass.
__device__ void stage_weights(const float* __restrict__ w, unsigned char* Wt, unsigned char* WTt, bool transposed) {
    const int sizes_n[5] = {kHid, kHid, kHid, kHid, kOut};
    int woff = 0, toff = 0;
    for (int l = 0; l < 5; ++l) {
        const int n = sizes_n[l], k = kHid;  // every layer has 64 inputs
        for (int e = threadIdx.x; e < n * k / 8; e += blockDim.x) {
            const int r = e / (k / 8), c0 = (e % (k / 8)) * 8;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = __ldg(w + woff + r * k + c0 + j);
            store8(Wt + toff, r, c0, k, v);
        }
        if (transposed) {
            for (int e = threadIdx.x; e < k * n / 8; e += blockDim.x) {  // W^T: k rows, n columns
                const int r = e / (n / 8), c0 = (e % (n / 8)) * 8;
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) v[j] = __ldg(w + woff + (c0 + j) * k + r);
                store8(WTt + toff, r, c0, n, v);
            }
        }
        woff += n * k;
        toff += n * k * 2;
    }
}
__host__ __device__ constexpr int wtile_off(int l) { return l * kHid * kHid * 2; }  // bytes; layer 4 is 16 x 64

// ---------------------------------------------------------------- kernels --
constexpr int kWBytes = 4 * kHid * kHid * 2 + kOut * kHid * 2;  // 34816
constexpr int kTileBytes = kTile * 64 * 2;                      // 16384

struct InferSmem {
    alignas(128) unsigned char W[kWBytes];
    alignas(128) unsigned char A[kTileBytes];
    alignas(8) unsigned long long bar;
    uint32_t tmem_slot;
    int fail;
};

enum : int { IN_GIVEN = 0, IN_ENCODE = 1, IN_RESOLVE = 2 };

// rows: n samples.  IN_GIVEN: inputs X [n,64], out [n,16].  IN_ENCODE: inputs
// encoded from (pos, dir), out = rgb [n,3].  IN_RESOLVE: as IN_ENCODE with a
// throughput W per row: out[row % npix] += scale * W * rgb (rows with W == 0
// are skipped).
template <int IN>
__global__ void __launch_bounds__(128) k_mlp_infer(Enc E, const float* __restrict__ w, const float* __restrict__ X,
                                                    const float* __restrict__ pos, const float* __restrict__ dir,
                                                    const float* __restrict__ thr, int64_t n, float* __restrict__ out,
                                                    int out_stride, int64_t npix, float scale) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    InferSmem& S = *reinterpret_cast<InferSmem*>(smem_align128(smem_raw));
    const int t = threadIdx.x;
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar)));
        S.fail = 0;
    }
    if (t < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_u32(&S.tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    stage_weights(w, S.W, nullptr, false);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    Engine G{S.tmem_slot, smem_u32(&S.bar), 0u, true};
    const int64_t tiles = (n + kTile - 1) / kTile;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t row = tile * kTile + t;
        float x[64];
        float3 Wr = f3(0.0f);
        bool live = row < n;
        if (IN == IN_RESOLVE && live) {
            Wr = ld3(thr + 3 * row);
            live = Wr.x != 0.0f || Wr.y != 0.0f || Wr.z != 0.0f;
        }
        if (live) {
            if (IN != IN_GIVEN) encode(E, ld3(pos + 3 * row), ld3(dir + 3 * row), x);
            else {
#pragma unroll
                for (int i = 0; i < 64; i += 4) {
                    float4 q = __ldg(reinterpret_cast<const float4*>(X + row * 64 + i));
                    x[i] = q.x; x[i + 1] = q.y; x[i + 2] = q.z; x[i + 3] = q.w;
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < 64; ++i) x[i] = 0.0f;
        }
        for (int layer = 0; layer < 5; ++layer) {
            const int nout = layer < 4 ? kHid : kOut;
#pragma unroll
            for (int k0 = 0; k0 < 64; k0 += 8) store8(S.A, t, k0, 64, x + k0);
            fence_async_smem();
            __syncthreads();
            if (S.fail) break;
            G.gemm(S.A, S.W + wtile_off(layer), nout, 64);
            G.read_row(nout, x);
            if (!G.ok) S.fail = 1;
            if (layer < 4) {
#pragma unroll
                for (int i = 0; i < 64; ++i) x[i] = fmaxf(x[i], 0.0f);
            }
            __syncthreads();  // every row is read before the tile is rewritten
        }
        if (S.fail) break;
        if (IN == IN_RESOLVE) {
            if (live) {
                float* o = out + 3 * (row % npix);
                atomicAdd(o + 0, scale * Wr.x * x[0]);
                atomicAdd(o + 1, scale * Wr.y * x[1]);
                atomicAdd(o + 2, scale * Wr.z * x[2]);
            }
        } else if (live) {
            for (int c = 0; c < out_stride; ++c) out[row * out_stride + c] = x[c];
        }
    }
    __syncthreads();
    if (S.fail && t == 0) {
        atomicOr(&g_cache_status, 1u << VRT_E_ITER_CAP);
        mbar_wait(G.bar, G.phase);  // bounded: the last issued MMA before its TMEM is freed
    }
    __syncthreads();
    if (t < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(S.tmem_slot));
}

struct TrainSmem {
    alignas(128) unsigned char W[kWBytes];
    alignas(128) unsigned char WT[kWBytes];
    alignas(128) unsigned char A[5][kTileBytes];   // layer inputs a0..a4 (BF16)
    alignas(128) unsigned char Gb[2][kTileBytes];  // backward tiles, ping-pong
    alignas(8) unsigned long long bar;
    uint32_t tmem_slot;
    int fail;
};

// dW_l[o][i] += sum_s G[s][o] A[s][i] over the tile (CUDA cores), atomically into wgrad
__device__ __forceinline__ void weight_grad(const unsigned char* G, int kg, const unsigned char* A, int nout,
                                            float* __restrict__ wgrad) {
    const int t = threadIdx.x;
    // thread t: output o, 64/(128/nout) inputs
    const int per_o = kTile / nout;             // threads per output row: 2 (nout 64) or 8 (nout 16)
    const int o = t / per_o, span = 64 / per_o;  // inputs per thread: 32 or 8
    const int i0 = (t % per_o) * span;
    float acc[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] = 0.0f;
    for (int s = 0; s < kTile; ++s) {
        const unsigned char* gp = G + core_off(s, o, kg);
        const float g = __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(gp));
        if (g == 0.0f) continue;
        for (int j = 0; j < span; j += 8) {
            float a[8];
            load8(A, s, i0 + j, 64, a);
#pragma unroll
            for (int q = 0; q < 8; ++q) acc[j + q] += g * a[q];
        }
    }
    for (int j = 0; j < span; ++j)
        if (acc[j] != 0.0f) atomicAdd(wgrad + o * 64 + i0 + j, acc[j]);
}

// One training pass over n samples: forward, relative L2 loss against target,
// backward into the encoding grid and the weights (gradients accumulate).
__global__ void __launch_bounds__(128) k_mlp_train(Enc E, const float* __restrict__ w, float* __restrict__ wgrad,
                                                    const float* __restrict__ pos, const float* __restrict__ dir,
                                                    const float* __restrict__ target, int64_t n, float inv_batch,
                                                    float* __restrict__ loss) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_align128(smem_raw));
    const int t = threadIdx.x;
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar)));
        S.fail = 0;
    }
    if (t < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_u32(&S.tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    stage_weights(w, S.W, S.WT, true);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    Engine G{S.tmem_slot, smem_u32(&S.bar), 0u, true};
    float lsum = 0.0f;
    const int64_t tiles = (n + kTile - 1) / kTile;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t row = tile * kTile + t;
        bool valid = row < n;
        float3 tg3 = f3(0.0f);
        if (valid) {  // rows without a finite target (a path that ended before the vertex) are skipped
            tg3 = ld3(target + 3 * row);
            valid = isfinite(tg3.x) && isfinite(tg3.y) && isfinite(tg3.z);
        }
        float3 p = f3(0.0f), d = make_float3(0.0f, 0.0f, 1.0f);
        float x[64];
        if (valid) {
            p = ld3(pos + 3 * row);
            d = ld3(dir + 3 * row);
            encode(E, p, d, x);
        } else {
#pragma unroll
            for (int i = 0; i < 64; ++i) x[i] = 0.0f;
        }
        // ---- forward, keeping every layer input
        for (int layer = 0; layer < 5; ++layer) {
            const int nout = layer < 4 ? kHid : kOut;
#pragma unroll
            for (int k0 = 0; k0 < 64; k0 += 8) store8(S.A[layer], t, k0, 64, x + k0);
            fence_async_smem();
            __syncthreads();
            if (S.fail) break;
            G.gemm(S.A[layer], S.W + wtile_off(layer), nout, 64);
            G.read_row(nout, x);
            if (!G.ok) S.fail = 1;
            if (layer < 4) {
#pragma unroll
                for (int i = 0; i < 64; ++i) x[i] = fmaxf(x[i], 0.0f);
            }
        }
        // ---- loss: relative L2, sum_c (y - t)^2 / (y^2 + 0.01), y detached in the denominator
        float g16[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) g16[i] = 0.0f;
        if (valid) {
            for (int c = 0; c < 3; ++c) {
                const float y = x[c], tg = c == 0 ? tg3.x : (c == 1 ? tg3.y : tg3.z);
                const float den = y * y + 0.01f;
                const float r = y - tg;
                lsum += r * r / den * inv_batch;
                g16[c] = 2.0f * r / den * inv_batch;
            }
        }
        // ---- backward: G5 = dL/dy (K = 16), then dH_l = G_{l+1} W_{l+1} on the tensor cores
        unsigned char* gcur = S.Gb[0];
        store8(gcur, t, 0, 16, g16);
        store8(gcur, t, 8, 16, g16 + 8);
        fence_async_smem();
        __syncthreads();
        if (S.fail) break;  // read after the barrier: every thread takes the same branch
        int kg = 16;
        for (int layer = 4; layer >= 0; --layer) {
            const int nout = layer < 4 ? kHid : kOut;
            // dX of this layer = G (128 x nout) * W_layer (nout x 64): B = W_layer^T (64 x nout)
            G.gemm(gcur, S.WT + wtile_off(layer), kHid, nout);
            weight_grad(gcur, kg, S.A[layer], nout, wgrad + layer * kHid * kHid);
            float dx[64];
            G.read_row(kHid, dx);
            if (!G.ok) S.fail = 1;
            if (layer > 0) {
                // through the ReLU that produced this layer's input
                float a[8];
#pragma unroll
                for (int k0 = 0; k0 < 64; k0 += 8) {
                    load8(S.A[layer], t, k0, 64, a);
#pragma unroll
                    for (int q = 0; q < 8; ++q) dx[k0 + q] = a[q] > 0.0f ? dx[k0 + q] : 0.0f;
                }
                unsigned char* gnext = (gcur == S.Gb[0]) ? S.Gb[1] : S.Gb[0];
                __syncthreads();  // weight_grad reads of gnext's previous contents are done
#pragma unroll
                for (int k0 = 0; k0 < 64; k0 += 8) store8(gnext, t, k0, 64, dx + k0);
                fence_async_smem();
                __syncthreads();
                gcur = gnext;
                kg = 64;
            } else if (valid) {
                // into the encoding grid: input 2l+f is a trilinear blend of level l's feature f
                float3 u = unit_coords(E, p);
                for (int l = 0; l < kLevels; ++l) {
                    const float g0 = dx[2 * l], g1 = dx[2 * l + 1];
                    if (g0 == 0.0f && g1 == 0.0f) continue;
                    Corner8 c;
                    level_corners(E, l, u, c);
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        atomicAdd(E.grid_grad + c.idx[k], c.wt[k] * g0);
                        atomicAdd(E.grid_grad + c.idx[k] + 1, c.wt[k] * g1);
                    }
                }
            }
            if (S.fail) break;
        }
        __syncthreads();
        if (S.fail) break;
    }
    // loss: warp sum, one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    if ((t & 31) == 0 && lsum != 0.0f) atomicAdd(loss, lsum);
    __syncthreads();
    if (S.fail && t == 0) {
        atomicOr(&g_cache_status, 1u << VRT_E_ITER_CAP);
        mbar_wait(G.bar, G.phase);  // bounded: the last issued MMA before its TMEM is freed
    }
    __syncthreads();
    if (t < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(S.tmem_slot));
}

// Adam (Kingma & Ba 2015) with bias correction; clears the gradient.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        g[i] = 0.0f;
    }
}

}  // namespace cache
}  // namespace vrt

// ------------------------------------------------------------------ C ABI --
using namespace vrt;
using namespace vrt::cache;

static int to_enc(const vrt_cache* c, Enc& E) {
    if (!c || !c->grid) return VRT_E_NULL_POINTER;
    if (c->levels != kLevels) return VRT_E_UNSUPPORTED;
    int64_t off = 0;
    for (int l = 0; l < kLevels; ++l) {
        if (c->res[l] < 1 || c->res[l] > 1024) return VRT_E_BAD_SHAPE;
        E.res[l] = c->res[l];
        E.off[l] = (int)off;
        off += (int64_t)(c->res[l] + 1) * (c->res[l] + 1) * (c->res[l] + 1) * 2;
        if (off >= (int64_t)INT32_MAX) return VRT_E_BAD_SHAPE;
    }
    E.grid = c->grid;
    E.grid_grad = c->grid_grad;
    E.bmin = make_float3(c->bmin[0], c->bmin[1], c->bmin[2]);
    E.inv_size = make_float3(1.0f / (c->bmax[0] - c->bmin[0]), 1.0f / (c->bmax[1] - c->bmin[1]),
                             1.0f / (c->bmax[2] - c->bmin[2]));
    return VRT_OK;
}

static int num_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// grid size for n samples, or 0 when the kernel cannot get its shared memory
template <class K>
static int mlp_blocks(K kernel, size_t smem, int64_t n, int per_sm) {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int64_t tiles = (n + kTile - 1) / kTile;
    int64_t blocks = (int64_t)num_sms() * per_sm;
    return (int)(tiles < blocks ? tiles : blocks);
}

extern "C" int64_t vrt_cache_grid_size(const int32_t res[16]) {
    int64_t off = 0;
    for (int l = 0; l < kLevels; ++l) off += (int64_t)(res[l] + 1) * (res[l] + 1) * (res[l] + 1) * 2;
    return off;
}

extern "C" int vrt_cache_mlp_fw(const float* weights, const float* inputs, int64_t n, float* out, void* stream) {
    if (n < 0) return VRT_E_BAD_SHAPE;
    if (n == 0) return VRT_OK;
    if (!weights || !inputs || !out) return VRT_E_NULL_POINTER;
    if (((uintptr_t)inputs & 15u) != 0) return VRT_E_INVALID_ARGUMENT;
    Enc E = {};
    size_t smem = sizeof(InferSmem) + 128;
    int blocks = mlp_blocks(k_mlp_infer<IN_GIVEN>, smem, n, 4);
    if (blocks <= 0) return VRT_E_CUDA;
    k_mlp_infer<IN_GIVEN><<<blocks, kTile, smem, (cudaStream_t)stream>>>(E, weights, inputs, nullptr, nullptr, nullptr,
                                                                         n, out, kOut, 0, 0.0f);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

extern "C" int vrt_cache_infer(const vrt_cache* c, const float* pos, const float* dir, int64_t n, float* rgb,
                               void* stream) {
    Enc E;
    int st = to_enc(c, E);
    if (st) return st;
    if (n < 0) return VRT_E_BAD_SHAPE;
    if (n == 0) return VRT_OK;
    if (!pos || !dir || !rgb || !c->weights) return VRT_E_NULL_POINTER;
    size_t smem = sizeof(InferSmem) + 128;
    int blocks = mlp_blocks(k_mlp_infer<IN_ENCODE>, smem, n, 4);
    if (blocks <= 0) return VRT_E_CUDA;
    k_mlp_infer<IN_ENCODE><<<blocks, kTile, smem, (cudaStream_t)stream>>>(E, c->weights, nullptr, pos, dir, nullptr, n,
                                                                          rgb, 3, 0, 0.0f);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

extern "C" int vrt_cache_resolve(const vrt_cache* c, const float* queries, int64_t n, int64_t npix, float scale,
                                 float* rgb, void* stream) {
    Enc E;
    int st = to_enc(c, E);
    if (st) return st;
    if (n < 0 || npix < 1) return VRT_E_BAD_SHAPE;
    if (n == 0) return VRT_OK;
    if (!queries || !rgb || !c->weights) return VRT_E_NULL_POINTER;
    size_t smem = sizeof(InferSmem) + 128;
    int blocks = mlp_blocks(k_mlp_infer<IN_RESOLVE>, smem, n, 4);
    if (blocks <= 0) return VRT_E_CUDA;
    k_mlp_infer<IN_RESOLVE><<<blocks, kTile, smem, (cudaStream_t)stream>>>(
        E, c->weights, nullptr, queries, queries + 3 * n, queries + 6 * n, n, rgb, 3, npix, scale);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

extern "C" int vrt_cache_train(const vrt_cache* c, const float* pos, const float* dir, const float* target, int64_t n,
                               float* loss, void* stream) {
    Enc E;
    int st = to_enc(c, E);
    if (st) return st;
    if (n < 0) return VRT_E_BAD_SHAPE;
    if (n == 0) return VRT_OK;
    if (!pos || !dir || !target || !loss || !c->weights || !c->weights_grad || !c->grid_grad) return VRT_E_NULL_POINTER;
    size_t smem = sizeof(TrainSmem) + 128;
    int blocks = mlp_blocks(k_mlp_train, smem, n, 1);
    if (blocks <= 0) return VRT_E_CUDA;
    k_mlp_train<<<blocks, kTile, smem, (cudaStream_t)stream>>>(E, c->weights, c->weights_grad, pos, dir, target, n,
                                                               1.0f / (float)n, loss);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

extern "C" int vrt_cache_adam(float* params, float* grads, float* m, float* v, int64_t n, float lr, float beta1,
                              float beta2, float eps, int32_t step, void* stream) {
    if (n < 0 || step < 1) return VRT_E_INVALID_ARGUMENT;
    if (n == 0) return VRT_OK;
    if (!params || !grads || !m || !v) return VRT_E_NULL_POINTER;
    float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    int64_t b = (n + 255) / 256;
    int blocks = (int)(b < 4096 ? b : 4096);
    k_adam<<<blocks, 256, 0, (cudaStream_t)stream>>>(params, grads, m, v, n, lr, beta1, beta2, eps, c1, c2);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

extern "C" int vrt_cache_status(void* stream) {
    if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return VRT_E_CUDA;
    uint32_t word = 0;
    if (cudaMemcpyFromSymbol(&word, g_cache_status, sizeof(word)) != cudaSuccess) return VRT_E_CUDA;
    if (word) {
        const uint32_t zero = 0;
        cudaMemcpyToSymbol(g_cache_status, &zero, sizeof(zero));
    }
    for (int code = 1; code < 32; ++code)
        if (word & (1u << code)) return code;
    return VRT_OK;
}
