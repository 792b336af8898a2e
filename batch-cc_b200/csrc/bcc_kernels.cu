// bcc_kernels.cu -- robot-independent kernels of the batch edge collision
// checker (sm_100a): the sample-offset scan, the environment code of the
// learned check order, shared-memory sizing, and the robot registry.  The
// robot-templated pipeline lives in bcc_pipeline.cuh and is instantiated once
// per robot in bcc_robot_<name>.cu.
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "bcc_device.cuh"
#include "bcc_kernels.h"
#include "bcc_mlp.h"

namespace bcc {

extern const RobotOps kPandaOps;
extern const RobotOps kFetchOps;
extern const RobotOps kBaxterOps;

const RobotOps* robot_ops(int robot) {
    switch (robot) {
        case 0: return &kPandaOps;
        case 1: return &kFetchOps;
        case 2: return &kBaxterOps;
        default: return nullptr;
    }
}

// ------------------------------------------------------------------ scan
// Single-CTA exclusive scan of 32*steps[e] into offs[e], offs[E] = total.
// Sums run in 64 bits and every offset saturates at INT32_MAX, so a total too
// large for the sample table can never wrap into a small, valid-looking one;
// the host rejects any total above its limit.
__global__ void scan_kernel(const int* __restrict__ steps, int E, int* __restrict__ offs) {
    __shared__ long long warp_sums[32];
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < E; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const long long v = (i < E) ? (long long)kLanes * steps[i] : 0;
        long long x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            long long w = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const long long warp_prefix = warp ? warp_sums[warp - 1] : 0;
        if (i < E) offs[i] = (int)min(carry + warp_prefix + x - v, 2147483647ll);
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += warp_prefix + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) offs[E] = (int)min(carry, 2147483647ll);
}

cudaError_t launch_scan(const int* steps, int E, int* offs, cudaStream_t st) {
    scan_kernel<<<1, 1024, 0, st>>>(steps, E, offs);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ sizing
// Dynamic shared memory of a check CTA: the largest environment's records plus,
// per warp, a (primitive, link) pair list of max_prims x groups entries, at
// most kPairCap.
size_t check_smem_bytes(int max_prims, int groups, size_t blob_smem, int warps) {
    const size_t ppw = (size_t)std::min((max_prims * groups + 7) & ~7, kPairCap);
    return blob_smem + (size_t)warps * ppw * sizeof(uint16_t);
}

size_t records_smem_bytes(int max_prims, int groups, int warps) {
    const size_t ppw = (size_t)((max_prims * groups + 7) & ~7);
    return (size_t)max_prims * kPrimF4 * 16 + (size_t)warps * ppw * sizeof(uint16_t);
}

// ------------------------------------------------------------------ environment code
// 32-value environment code (one warp per environment): [0..3] counts of
// sphere-like, capsule-like and box-like primitives and the total, / 64;
// [4..27] for 8 fixed anchor points the distance from the anchor to the
// nearest primitive of each of the three kinds (clamped to [-0.5, 1.5] m);
// [28..31] mean primitive centre xyz and mean extent.
__device__ __forceinline__ float prim_point_dist(const float4* rec, float x, float y, float z) {
    const float4 w0 = rec[0], w1 = rec[1], w2 = rec[2], w3 = rec[3];
    const float dx = x - w0.x, dy = y - w0.y, dz = z - w0.z;
    const float e1 = fmaxf(fabsf(w1.x * dx + w1.y * dy + w1.z * dz) - w1.w, 0.0f);
    const float e2 = fmaxf(fabsf(w2.x * dx + w2.y * dy + w2.z * dz) - w2.w, 0.0f);
    const float e3 = fmaxf(fabsf(w3.x * dx + w3.y * dy + w3.z * dz) - w3.w, 0.0f);
    return sqrtf(e1 * e1 + e2 * e2 + e3 * e3) - w0.w;
}

__global__ void env_encode_kernel(const float4* __restrict__ blobs, const float4* __restrict__ hdr, int N,
                                  float* __restrict__ code) {
    const int env = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (env >= N) return;
    const float4 h0 = hdr[2 * env], h1 = hdr[2 * env + 1];
    const float4* rec = blobs + __float_as_uint(h0.w);
    const int np = (int)(__float_as_uint(h1.w) & 0xffffu);
    float cnt[3] = {0, 0, 0}, best[8][3], mean[4] = {0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < 8; ++a) best[a][0] = best[a][1] = best[a][2] = 1.5f;
    for (int p = lane; p < np; p += 32) {
        const float4* r = rec + p * kPrimF4;
        const float4 w0 = r[0];
        const float hsum = r[1].w + r[2].w + r[3].w;
        const int kind = w0.w > 0.0f ? (hsum > 0.0f ? 1 : 0) : 2;  // sphere, capsule, box
        cnt[kind] += 1.0f;
        mean[0] += w0.x;
        mean[1] += w0.y;
        mean[2] += w0.z;
        mean[3] += w0.w + hsum;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const float ax = (a & 1) ? 0.35f : -0.35f, ay = (a & 2) ? 0.35f : -0.35f, az = (a & 4) ? 0.8f : 0.3f;
            best[a][kind] = fminf(best[a][kind], prim_point_dist(r, ax, ay, az));
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) cnt[k] += __shfl_xor_sync(0xffffffffu, cnt[k], o);
#pragma unroll
        for (int k = 0; k < 4; ++k) mean[k] += __shfl_xor_sync(0xffffffffu, mean[k], o);
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int k = 0; k < 3; ++k) best[a][k] = fminf(best[a][k], __shfl_xor_sync(0xffffffffu, best[a][k], o));
    }
    if (lane == 0) {
        float* c = code + (size_t)env * kEnvCode;
        c[0] = cnt[0] / 64.0f;
        c[1] = cnt[1] / 64.0f;
        c[2] = cnt[2] / 64.0f;
        c[3] = (float)np / 64.0f;
        for (int a = 0; a < 8; ++a)
            for (int k = 0; k < 3; ++k) c[4 + a * 3 + k] = fminf(fmaxf(best[a][k], -0.5f), 1.5f);
        const float inv = np > 0 ? 1.0f / (float)np : 0.0f;
        for (int k = 0; k < 4; ++k) c[28 + k] = mean[k] * inv;
    }
}

cudaError_t launch_env_encode(const float4* blobs, const float4* env_hdr, int num_envs, float* code, cudaStream_t st) {
    if (num_envs <= 0) return cudaSuccess;
    env_encode_kernel<<<(num_envs * 32 + 255) / 256, 256, 0, st>>>(blobs, env_hdr, num_envs, code);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ training rows
__global__ void gather_rows_kernel(const uint4* __restrict__ x, const uint8_t* __restrict__ y,
                                   const int* __restrict__ perm, int rows, uint4* __restrict__ x2,
                                   uint8_t* __restrict__ y2) {
    constexpr int W = kMlpIn * 2 / 16;  // uint4 words per row
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const int src = perm[i];
#pragma unroll
    for (int w = 0; w < W; ++w) x2[(size_t)i * W + w] = x[(size_t)src * W + w];
    y2[i] = y[src];
}

cudaError_t launch_gather_rows(const uint16_t* x, const uint8_t* y, const int* perm, int rows, uint16_t* x2,
                               uint8_t* y2, cudaStream_t st) {
    static_assert(kMlpIn * 2 % 16 == 0, "feature rows are whole 16-byte words");
    if (rows <= 0) return cudaSuccess;
    gather_rows_kernel<<<(rows + 255) / 256, 256, 0, st>>>(reinterpret_cast<const uint4*>(x), y, perm, rows,
                                                           reinterpret_cast<uint4*>(x2), y2);
    return cudaGetLastError();
}

}  // namespace bcc
