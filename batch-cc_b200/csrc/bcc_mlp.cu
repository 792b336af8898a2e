// bcc_mlp.cu -- the collision-likelihood MLP on 5th-generation tensor cores.
//
// Network (per sample configuration in one environment):
//     x (48 = 7 normalised joints + 32 environment code + 9 zero) -> 128 -> 128 -> 128 -> 1
// ReLU between layers, logit output.  Weights and activations are BF16 in
// shared memory (core-matrix images, see bcc_tc.cuh), products accumulate in
// FP32 tensor memory via tcgen05.mma (M = 128 rows per tile, N = 128), the
// epilogues (bias, ReLU, final 128-wide dot product) run in FP32 registers.
//
// Parameters (FP32 masters, flat, kMlpParams floats):
//     W1 [48][128] (in x out), b1 [128], W2 [128][128], b2 [128],
//     W3 [128][128], b3 [128], w4 [128], b4 [1]
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/bcc.h"
#include "bcc_ctx.h"
#include "bcc_device.cuh"
#include "bcc_mlp.h"
#include "bcc_tc.cuh"

namespace bcc {

// Offsets of the parameter blocks in the flat FP32 vector.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpIn * kMlpHidden;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpHidden * kMlpHidden;
constexpr int kOffW4 = kOffB3 + kMlpHidden;
constexpr int kOffB4 = kOffW4 + kMlpHidden;
static_assert(kOffB4 + 1 == kMlpParams, "parameter layout");

// Images (BF16 core-matrix layouts, bcc_tc.cuh): W1^T [128][48] -- its column
// 47 carries b1, the forward kernel reads feature 47 as 1 --, W2^T, W3^T
// [128][128] (the training kernel uses these three), then for the forward
// kernel only: W4 [16][128] (row 0 = w4, the last layer as an N = 16 MMA) and
// B2, B3 [128][16] (column 0 = b2 / b3, added by one K = 16 MMA against a
// ones column).
constexpr uint32_t kImgW1 = kMlpHidden * kMlpIn * 2;       // 12288
constexpr uint32_t kImgW = kMlpHidden * kMlpHidden * 2;    // 32768
constexpr uint32_t kImgSmall = kMlpHidden * 16 * 2;         // 4096: W4, B2, B3 and the ones image
constexpr uint32_t kImagesW = kImgW1 + 2 * kImgW;           // W1T | W2T | W3T
constexpr uint32_t kImagesBytes = kImagesW + 3 * kImgSmall;  // ... | W4 | B2 | B3
constexpr int kBiasCol = kMlpIn - 1;                        // feature 47: reserved, read as 1 by the forward kernel

// Shared-memory map of the forward kernel (bytes): the images, the ones image
// (A operand of the bias MMAs), then per row group one buffer for its X tile
// (128 x 48) and, once the first MMA has consumed X, its H tile (128 x 128),
// b4, the groups' mbarriers and the TMEM address slot.
constexpr uint32_t kSmW1 = 0;
constexpr uint32_t kSmW2 = kSmW1 + kImgW1;
constexpr uint32_t kSmW3 = kSmW2 + kImgW;
constexpr uint32_t kSmW4 = kSmW3 + kImgW;
constexpr uint32_t kSmB2 = kSmW4 + kImgSmall;
constexpr uint32_t kSmB3 = kSmB2 + kImgSmall;
constexpr uint32_t kSmOnes = kSmB3 + kImgSmall;
constexpr int kFwdGroups = 4;                              // independent 128-row tile streams per CTA
constexpr uint32_t kFwdTmemCols = 512;                     // power of two >= 128 x groups
// Group g's buffer at kSmGroup0 + g * stride holds its X tile (128 x 48) until
// the first layer's MMA has read it, then its H tile (128 x 128).
constexpr uint32_t kSmGroup0 = kSmOnes + kImgSmall;
constexpr uint32_t kSmGroupStride = kImgW;
constexpr uint32_t kSmVec = kSmGroup0 + kFwdGroups * kSmGroupStride;  // b4
constexpr uint32_t kSmBar = kSmVec + 16;
constexpr uint32_t kSmTmem = kSmBar + 8 * kFwdGroups;
constexpr uint32_t kFwdSmem = kSmTmem + 8;
static_assert(kSmGroup0 % 16 == 0 && kSmGroupStride % 16 == 0, "core-matrix images are 16-byte aligned");
static_assert(kSmW4 == kImagesW && kSmOnes == kImagesBytes, "forward images are copied as one block");
static_assert(kFwdSmem <= 227 * 1024, "forward kernel shared memory");

// ---------------------------------------------------------------- images
// FP32 masters -> BF16 core-matrix images of W1^T [128][48], W2^T, W3^T.
// Feature 47 is zero in every input row, so W1's row 47 never contributes;
// the image's column 47 holds b1 instead, which the forward kernel adds by
// reading feature 47 as 1 (the training kernel reads it as the 0 it is and
// adds b1 in its epilogue).
__global__ void mlp_pack_kernel(const float* __restrict__ params, uint8_t* __restrict__ images) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n1 = kMlpHidden * kMlpIn, n2 = kMlpHidden * kMlpHidden, ns = kMlpHidden * 16;
    if (i < n1) {
        const int out = i / kMlpIn, in = i % kMlpIn;
        const float w = in == kBiasCol ? params[kOffB1 + out] : params[kOffW1 + in * kMlpHidden + out];
        *reinterpret_cast<__nv_bfloat16*>(images + tc::cm_offset(out, in, kMlpIn)) = __float2bfloat16_rn(w);
    } else if (i < n1 + 2 * n2) {
        const int j = i - n1;
        const int layer = j / n2, r = j % n2;
        const int out = r / kMlpHidden, in = r % kMlpHidden;
        const float w = params[(layer ? kOffW3 : kOffW2) + in * kMlpHidden + out];
        *reinterpret_cast<__nv_bfloat16*>(images + kImgW1 + layer * kImgW + tc::cm_offset(out, in, kMlpHidden)) =
            __float2bfloat16_rn(w);
    } else if (i < n1 + 2 * n2 + ns) {  // W4 [16][128]: row 0 = w4
        const int j = i - n1 - 2 * n2;
        const int out = j / kMlpHidden, in = j % kMlpHidden;
        const float w = out == 0 ? params[kOffW4 + in] : 0.0f;
        *reinterpret_cast<__nv_bfloat16*>(images + kImagesW + tc::cm_offset(out, in, kMlpHidden)) =
            __float2bfloat16_rn(w);
    } else if (i < n1 + 2 * n2 + 3 * ns) {  // B2, B3 [128][16]: column 0 = bias
        const int j = i - n1 - 2 * n2 - ns;
        const int layer = j / ns, r = j % ns;
        const int out = r / 16, in = r % 16;
        const float w = in == 0 ? params[(layer ? kOffB3 : kOffB2) + out] : 0.0f;
        *reinterpret_cast<__nv_bfloat16*>(images + kImagesW + (1 + layer) * kImgSmall + tc::cm_offset(out, in, 16)) =
            __float2bfloat16_rn(w);
    }
}

// ---------------------------------------------------------------- forward
// ReLU of two FP32 values, rounded to BF16 and packed (lo in the low half).
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// Forward epilogue of a hidden layer whose bias the MMAs already added: this
// thread's accumulator row, ReLU, BF16 into the H image (one conversion per
// two values).  Two 16-column loads are in flight before each wait.
__device__ __forceinline__ void epilogue_relu_only(uint32_t taddr, uint8_t* himg, int row) {
#pragma unroll 1
    for (int c0 = 0; c0 < kMlpHidden; c0 += 32) {
        float v[32];
        tc::tmem_ld16(taddr + c0, v);
        tc::tmem_ld16(taddr + c0 + 16, v + 16);
        tc::wait_ld();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint4 w;
            w.x = relu_bf16x2(v[8 * q + 0], v[8 * q + 1]);
            w.y = relu_bf16x2(v[8 * q + 2], v[8 * q + 3]);
            w.z = relu_bf16x2(v[8 * q + 4], v[8 * q + 5]);
            w.w = relu_bf16x2(v[8 * q + 6], v[8 * q + 7]);
            *reinterpret_cast<uint4*>(himg + tc::cm_offset(row, c0 + 8 * q, kMlpHidden)) = w;
        }
    }
}

// Bias + ReLU of one 128-column accumulator row (this thread's row), written as
// BF16 into the H image; `taddr` = TMEM address of column 0 of this warp's lanes.
// One warp group's epilogue of a hidden layer: TMEM accumulator row + bias, ReLU,
// BF16 into the H image.  Two 16-column loads are in flight before each wait.
__device__ __forceinline__ void epilogue_relu_to_smem(uint32_t taddr, const float* bias, uint8_t* himg, int row) {
#pragma unroll 1
    for (int c0 = 0; c0 < kMlpHidden; c0 += 32) {
        float v[32];
        tc::tmem_ld16(taddr + c0, v);
        tc::tmem_ld16(taddr + c0 + 16, v + 16);
        tc::wait_ld();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint32_t packed[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float a = fmaxf(v[16 * h + 2 * i] + bias[c0 + 16 * h + 2 * i], 0.0f);
                const float b = fmaxf(v[16 * h + 2 * i + 1] + bias[c0 + 16 * h + 2 * i + 1], 0.0f);
                __nv_bfloat162 hh = __floats2bfloat162_rn(a, b);
                packed[i] = *reinterpret_cast<uint32_t*>(&hh);
            }
            *reinterpret_cast<uint4*>(himg + tc::cm_offset(row, c0 + 16 * h, kMlpHidden)) =
                make_uint4(packed[0], packed[1], packed[2], packed[3]);
            *reinterpret_cast<uint4*>(himg + tc::cm_offset(row, c0 + 16 * h + 8, kMlpHidden)) =
                make_uint4(packed[4], packed[5], packed[6], packed[7]);
        }
    }
}

// Barrier of one 128-thread warp group (named barrier 1 + group).
__device__ __forceinline__ void group_sync(int grp) {
    asm volatile("bar.sync %0, 128;" ::"r"(1 + grp) : "memory");
}

// Barrier of one warp group that also ORs a predicate over its threads.
__device__ __forceinline__ bool group_sync_or(bool pred, int grp) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(1 + grp)
        : "memory");
    return r != 0;
}

// Persistent: each CTA loads the weights once; its four warp groups (4 warps,
// one row per thread each) run independent streams of 128-row tiles, each with
// its own X/H buffer, TMEM accumulator (columns 128 g ..) and mbarrier, so one
// group's MMAs overlap the others' epilogues (all 512 TMEM columns in use).  The biases ride in the MMAs (b1
// as column 47 of W1^T against feature 47 read as 1; b2, b3 by a K = 16 MMA of
// a ones column against B2 / B3) and the output layer is an N = 16 MMA against
// W4, so each hidden epilogue is only ReLU + BF16 conversion + store.  x: BF16
// [rows][48] row-major (feature 47 zero); logits: FP32 [rows].
__global__ void __launch_bounds__(128 * kFwdGroups, 1)
    mlp_forward_kernel(const uint16_t* __restrict__ x, int rows, const int* __restrict__ rows_dev,
                       const uint4* __restrict__ images, const float* __restrict__ params, float* __restrict__ logits,
                       int* __restrict__ err) {
    // rows_dev (optional): the row count produced on the device, capped by rows.
    if (rows_dev) rows = min(rows, *rows_dev);
    // The grid is sized for the host's row bound; CTAs without a tile of the
    // device count leave before loading the weights.
    if ((long long)blockIdx.x * kFwdGroups * 128 >= (long long)rows) return;
    extern __shared__ __align__(1024) uint8_t sm[];
    const int t = threadIdx.x, warp = t >> 5, grp = t >> 7, gt = t & 127;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmBar) + grp;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kSmTmem);
    float* vec = reinterpret_cast<float*>(sm + kSmVec);
    uint8_t* xs = sm + kSmGroup0 + grp * kSmGroupStride;
    uint8_t* hs = xs;  // H overwrites X once the first layer's MMA has read it

    for (uint32_t i = t; i < kImagesBytes / 16; i += blockDim.x) reinterpret_cast<uint4*>(sm)[i] = images[i];
    if (t < 128) {  // ones image [128][16]: column 0 = 1 (BF16 0x3f80), the rest 0
        *reinterpret_cast<uint4*>(sm + kSmOnes + tc::cm_offset(t, 0, 16)) = make_uint4(0x3f80u, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(sm + kSmOnes + tc::cm_offset(t, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
    }
    if (t == 0) {
        vec[0] = params[kOffB4];
        for (int g = 0; g < kFwdGroups; ++g) mbar_init(reinterpret_cast<uint64_t*>(sm + kSmBar) + g, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, kFwdTmemCols);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tmem_slot + 128u * grp;
    const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const uint32_t idesc = tc::make_idesc_bf16(128, kMlpHidden, 0, 0);
    const uint32_t idesc16 = tc::make_idesc_bf16(128, 16, 0, 0);
    const uint32_t sbase = tc::smem_addr(sm);
    const float b4 = vec[0];
    uint32_t phase = 0;
    bool bad = false;

    const int tiles = (rows + 127) / 128;
    const int tile_step = gridDim.x * kFwdGroups;
    // X rows are loaded one tile ahead into registers, so their latency overlaps
    // the current tile's layers.
    uint4 xv[kMlpIn / 8];
    auto load_x = [&](int tile) {
        const int row = tile * 128 + gt;
        const uint4* src = reinterpret_cast<const uint4*>(x + (size_t)row * kMlpIn);
#pragma unroll
        for (int j = 0; j < kMlpIn / 8; ++j) xv[j] = (tile < tiles && row < rows) ? src[j] : make_uint4(0, 0, 0, 0);
    };
    static_assert(kBiasCol == kMlpIn - 1, "the bias feature is the last of the row's last 16-byte chunk");
    load_x(blockIdx.x * kFwdGroups + grp);
    for (int tile = blockIdx.x * kFwdGroups + grp; tile < tiles && !bad; tile += tile_step) {
        const int row = tile * 128 + gt;
        // X tile: this thread's row, six 16-byte chunks of 8 features; feature 47
        // (zero in the input) is read as 1 to pick up b1 from W1^T's column 47.
        xv[kMlpIn / 8 - 1].w = (xv[kMlpIn / 8 - 1].w & 0xffffu) | 0x3f800000u;
#pragma unroll
        for (int j = 0; j < kMlpIn / 8; ++j) *reinterpret_cast<uint4*>(xs + tc::cm_offset(gt, 8 * j, kMlpIn)) = xv[j];
        load_x(tile + tile_step);
        // Four MMA stages (three hidden layers, the output layer): MMAs from the
        // group's first thread, epilogue from all.
#pragma unroll 1
        for (int layer = 0; layer < 4; ++layer) {
            tc::fence_async_smem();
            tc::fence_before();
            group_sync(grp);
            if (gt == 0) {
                tc::fence_after();
                if (layer == 0) {
                    const uint32_t a0 = tc::smem_addr(xs), b0 = sbase + kSmW1;
                    constexpr uint32_t sbo = (uint32_t)(kMlpIn / 8) * 128u;
                    for (int s = 0; s < kMlpIn / 16; ++s)
                        tc::mma_bf16(tmem, tc::make_desc(a0 + 256u * s, 128u, sbo),
                                     tc::make_desc(b0 + 256u * s, 128u, sbo), idesc, s > 0 ? 1u : 0u);
                } else {
                    const uint32_t a0 = tc::smem_addr(hs);
                    const uint32_t b0 = sbase + (layer == 1 ? kSmW2 : layer == 2 ? kSmW3 : kSmW4);
                    constexpr uint32_t sbo = (uint32_t)(kMlpHidden / 8) * 128u;
                    for (int s = 0; s < kMlpHidden / 16; ++s)
                        tc::mma_bf16(tmem, tc::make_desc(a0 + 256u * s, 128u, sbo),
                                     tc::make_desc(b0 + 256u * s, 128u, sbo), layer == 3 ? idesc16 : idesc,
                                     s > 0 ? 1u : 0u);
                    if (layer < 3)  // + bias: ones [128][16] x B [128][16]^T
                        tc::mma_bf16(tmem, tc::make_desc(sbase + kSmOnes, 128u, 256u),
                                     tc::make_desc(sbase + (layer == 1 ? kSmB2 : kSmB3), 128u, 256u), idesc, 1u);
                }
                tc::commit(bar);
            }
            const bool ok = mbar_wait_bounded(bar, phase, 1u << 22);
            if (group_sync_or(!ok, grp)) {  // group-uniform decision
                bad = true;
                break;
            }
            phase ^= 1u;
            tc::fence_after();
            if (layer < 3) {
                epilogue_relu_only(taddr, hs, gt);
            } else {
                const float z = tc::tmem_ld1(taddr);
                tc::wait_ld();
                if (row < rows) logits[row] = z + b4;
            }
        }
    }
    if (bad && gt == 0) atomicOr(err, 1);
    if (bad) mbar_wait_bounded(bar, phase, 1u << 22);  // let in-flight MMAs finish before freeing TMEM
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0) tc::tmem_free(*tmem_slot, kFwdTmemCols);
}

// ---------------------------------------------------------------- training
// One CTA (128 threads, one row per thread) runs forward and backward over its
// 128-row tiles.  Activations stay in shared memory as BF16 images; the three
// weight-gradient accumulators stay in tensor memory across tiles and are
// added to the global FP32 gradient once at the end.  Loss: mean binary
// cross-entropy of the logit against the 0/1 label (scale = 1 / total rows).
//
// GEMMs (M = 128 unless noted; "K" / "MN" = operand read K- or MN-major):
//   forward   z1 = X W1 (A=X K, B=W1T K), z2 = H1 W2, z3 = H2 W3
//   backward  dW3 += H2^T dZ3   (A=H2 MN, B=dZ3 MN, K = rows)
//             dH2  = dZ3 W3^T   (A=dZ3 K, B=W3T MN)
//             dW2 += H1^T dZ2,  dH1 = dZ2 W2^T
//             dW1^T += dZ1^T X  (A=dZ1 MN, B=X MN, N = 48)
constexpr uint32_t kTrW1 = 0;
constexpr uint32_t kTrW2 = kTrW1 + kImgW1;
constexpr uint32_t kTrW3 = kTrW2 + kImgW;
constexpr uint32_t kTrX = kTrW3 + kImgW;
constexpr uint32_t kTrH1 = kTrX + kImgW1;
constexpr uint32_t kTrH2 = kTrH1 + kImgW;
constexpr uint32_t kTrD = kTrH2 + kImgW;
constexpr uint32_t kTrVec = kTrD + kImgW;                 // b1 b2 b3 w4 b4 (params)
constexpr uint32_t kTrGrad = kTrVec + 5 * kMlpHidden * 4;  // db1 db2 db3 dw4 db4 loss
constexpr uint32_t kTrBar = kTrGrad + 5 * kMlpHidden * 4 + 16;
constexpr uint32_t kTrTmem = kTrBar + 8;
constexpr uint32_t kTrainSmem = kTrTmem + 8;
// TMEM columns: forward / backward-data accumulator, dW3, dW2, dW1^T.
constexpr uint32_t kColAcc = 0, kColW3 = 128, kColW2 = 256, kColW1 = 384;

__device__ __forceinline__ void gemm_issue(uint32_t d, uint32_t a0, uint32_t a_lbo, uint32_t a_sbo, uint32_t a_step,
                                           uint32_t b0, uint32_t b_lbo, uint32_t b_sbo, uint32_t b_step, int ksteps,
                                           uint32_t idesc, bool accumulate) {
    for (int s = 0; s < ksteps; ++s)
        tc::mma_bf16(d, tc::make_desc(a0 + a_step * s, a_lbo, a_sbo), tc::make_desc(b0 + b_step * s, b_lbo, b_sbo),
                     idesc, (accumulate || s > 0) ? 1u : 0u);
}

// Column sums over the CTA's 128 rows of per-row values v[0..15] (columns
// c0..c0+15), added into acc[c0 + i] in shared memory.
__device__ __forceinline__ void colsum16(const float* v, float* acc, int c0) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        float x = v[i];
#pragma unroll
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == i) atomicAdd(acc + c0 + i, x);
    }
}

__device__ __forceinline__ float bf16_at(const uint8_t* img, int r, int c, int K) {
    return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(img + tc::cm_offset(r, c, K)));
}

__global__ void __launch_bounds__(128, 1)
    mlp_train_kernel(const uint16_t* __restrict__ x, const uint8_t* __restrict__ y, int rows,
                     const uint4* __restrict__ images, const float* __restrict__ params, float* __restrict__ grads,
                     float* __restrict__ loss_sum, int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int t = threadIdx.x, warp = t >> 5;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kTrBar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kTrTmem);
    float* vec = reinterpret_cast<float*>(sm + kTrVec);    // b1 | b2 | b3 | w4 | b4
    float* gv = reinterpret_cast<float*>(sm + kTrGrad);    // db1 | db2 | db3 | dw4 | db4, loss
    const float inv_rows = 1.0f / (float)rows;

    for (uint32_t i = t; i < kImagesW / 16; i += blockDim.x) reinterpret_cast<uint4*>(sm)[i] = images[i];
    for (int i = t; i < kMlpHidden; i += blockDim.x) {
        vec[i] = params[kOffB1 + i];
        vec[kMlpHidden + i] = params[kOffB2 + i];
        vec[2 * kMlpHidden + i] = params[kOffB3 + i];
        vec[3 * kMlpHidden + i] = params[kOffW4 + i];
    }
    for (int i = t; i < 5 * kMlpHidden + 4; i += blockDim.x) gv[i] = 0.0f;
    if (t == 0) {
        vec[4 * kMlpHidden] = params[kOffB4];
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(tmem_slot, 512);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_off = (uint32_t)(32 * warp) << 16;
    const uint32_t sb = tc::smem_addr(sm);
    const uint32_t id_fwd = tc::make_idesc_bf16(128, 128, 0, 0);   // A K-major, B K-major
    const uint32_t id_dw = tc::make_idesc_bf16(128, 128, 1, 1);    // A MN, B MN
    const uint32_t id_dh = tc::make_idesc_bf16(128, 128, 0, 1);    // A K, B MN
    const uint32_t id_dw1 = tc::make_idesc_bf16(128, 48, 1, 1);    // dW1^T: N = 48
    uint32_t phase = 0;
    bool bad = false, first = true;
    float* db1 = gv;
    float* db2 = gv + kMlpHidden;
    float* db3 = gv + 2 * kMlpHidden;
    float* dw4 = gv + 3 * kMlpHidden;

    // Issue (thread 0) + wait (all): returns false on a timed-out wait.
    auto sync_issue = [&](auto&& issue) -> bool {
        tc::fence_async_smem();
        tc::fence_before();
        __syncthreads();
        if (t == 0) {
            tc::fence_after();
            issue();
            tc::commit(bar);
        }
        const bool ok = mbar_wait_bounded(bar, phase, 1u << 22);
        if (__syncthreads_or(!ok)) return false;
        phase ^= 1u;
        tc::fence_after();
        return true;
    };

    const int tiles = (rows + 127) / 128;
    for (int tile = blockIdx.x; tile < tiles && !bad; tile += gridDim.x) {
        const int row = tile * 128 + t;
        const bool live = row < rows;
        const uint4* src = reinterpret_cast<const uint4*>(x + (size_t)row * kMlpIn);
#pragma unroll
        for (int j = 0; j < kMlpIn / 8; ++j)
            *reinterpret_cast<uint4*>(sm + kTrX + tc::cm_offset(t, 8 * j, kMlpIn)) = live ? src[j] : make_uint4(0, 0, 0, 0);
        const float label = live ? (float)y[row] : 0.0f;

        // ---- forward
        if (!sync_issue([&] { gemm_issue(tmem + kColAcc, sb + kTrX, 128, 768, 256, sb + kTrW1, 128, 768, 256, 3, id_fwd, false); })) { bad = true; break; }
        epilogue_relu_to_smem(tmem + lane_off + kColAcc, vec, sm + kTrH1, t);
        if (!sync_issue([&] { gemm_issue(tmem + kColAcc, sb + kTrH1, 128, 2048, 256, sb + kTrW2, 128, 2048, 256, 8, id_fwd, false); })) { bad = true; break; }
        epilogue_relu_to_smem(tmem + lane_off + kColAcc, vec + kMlpHidden, sm + kTrH2, t);
        if (!sync_issue([&] { gemm_issue(tmem + kColAcc, sb + kTrH2, 128, 2048, 256, sb + kTrW3, 128, 2048, 256, 8, id_fwd, false); })) { bad = true; break; }
        float logit = vec[4 * kMlpHidden];
#pragma unroll 1
        for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + lane_off + kColAcc + c0, v);
            tc::wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) logit = fmaf(fmaxf(v[i] + vec[2 * kMlpHidden + c0 + i], 0.0f), vec[3 * kMlpHidden + c0 + i], logit);
        }
        // ---- loss and dlogit (mean BCE)
        const float prob = 1.0f / (1.0f + __expf(-logit));
        const float dlogit = live ? (prob - label) * inv_rows : 0.0f;
        const float l = live ? (fmaxf(logit, 0.0f) - logit * label + log1pf(__expf(-fabsf(logit)))) : 0.0f;
        {
            float s1 = l, s2 = dlogit;
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                s1 += __shfl_xor_sync(0xffffffffu, s1, o);
                s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            }
            if ((t & 31) == 0) {
                atomicAdd(gv + 5 * kMlpHidden + 1, s1);
                atomicAdd(gv + 4 * kMlpHidden, s2);
            }
        }
        // dz3 = dlogit * w4 * (h3 > 0); dw4 += dlogit * h3; db3 += dz3
#pragma unroll 1
        for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
            float v[16], g3[16], gw[16];
            tc::tmem_ld16(tmem + lane_off + kColAcc + c0, v);
            tc::wait_ld();
            uint32_t packed[8];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float h3 = fmaxf(v[i] + vec[2 * kMlpHidden + c0 + i], 0.0f);
                gw[i] = dlogit * h3;
                g3[i] = h3 > 0.0f ? dlogit * vec[3 * kMlpHidden + c0 + i] : 0.0f;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                __nv_bfloat162 h = __floats2bfloat162_rn(g3[2 * i], g3[2 * i + 1]);
                packed[i] = *reinterpret_cast<uint32_t*>(&h);
            }
            *reinterpret_cast<uint4*>(sm + kTrD + tc::cm_offset(t, c0, kMlpHidden)) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            *reinterpret_cast<uint4*>(sm + kTrD + tc::cm_offset(t, c0 + 8, kMlpHidden)) = make_uint4(packed[4], packed[5], packed[6], packed[7]);
            colsum16(gw, dw4, c0);
            colsum16(g3, db3, c0);
        }
        // ---- dW3 += H2^T dZ3 ; dH2 = dZ3 W3^T
        const bool acc_w = !first;
        if (!sync_issue([&] {
                gemm_issue(tmem + kColW3, sb + kTrH2, 2048, 128, 4096, sb + kTrD, 2048, 128, 4096, 8, id_dw, acc_w);
                gemm_issue(tmem + kColAcc, sb + kTrD, 128, 2048, 256, sb + kTrW3, 2048, 128, 4096, 8, id_dh, false);
            })) { bad = true; break; }
        // dz2 = dh2 * (h2 > 0) -> D ; db2 += dz2
#pragma unroll 1
        for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + lane_off + kColAcc + c0, v);
            tc::wait_ld();
            uint32_t packed[8];
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = bf16_at(sm + kTrH2, t, c0 + i, kMlpHidden) > 0.0f ? v[i] : 0.0f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                packed[i] = *reinterpret_cast<uint32_t*>(&h);
            }
            *reinterpret_cast<uint4*>(sm + kTrD + tc::cm_offset(t, c0, kMlpHidden)) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            *reinterpret_cast<uint4*>(sm + kTrD + tc::cm_offset(t, c0 + 8, kMlpHidden)) = make_uint4(packed[4], packed[5], packed[6], packed[7]);
            colsum16(v, db2, c0);
        }
        // ---- dW2 += H1^T dZ2 ; dH1 = dZ2 W2^T
        if (!sync_issue([&] {
                gemm_issue(tmem + kColW2, sb + kTrH1, 2048, 128, 4096, sb + kTrD, 2048, 128, 4096, 8, id_dw, acc_w);
                gemm_issue(tmem + kColAcc, sb + kTrD, 128, 2048, 256, sb + kTrW2, 2048, 128, 4096, 8, id_dh, false);
            })) { bad = true; break; }
#pragma unroll 1
        for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + lane_off + kColAcc + c0, v);
            tc::wait_ld();
            uint32_t packed[8];
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = bf16_at(sm + kTrH1, t, c0 + i, kMlpHidden) > 0.0f ? v[i] : 0.0f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                packed[i] = *reinterpret_cast<uint32_t*>(&h);
            }
            *reinterpret_cast<uint4*>(sm + kTrD + tc::cm_offset(t, c0, kMlpHidden)) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            *reinterpret_cast<uint4*>(sm + kTrD + tc::cm_offset(t, c0 + 8, kMlpHidden)) = make_uint4(packed[4], packed[5], packed[6], packed[7]);
            colsum16(v, db1, c0);
        }
        // ---- dW1^T += dZ1^T X
        if (!sync_issue([&] {
                gemm_issue(tmem + kColW1, sb + kTrD, 2048, 128, 4096, sb + kTrX, 768, 128, 1536, 8, id_dw1, acc_w);
            })) { bad = true; break; }
        first = false;
    }
    if (bad) {
        if (t == 0) atomicOr(err, 1);
        mbar_wait_bounded(bar, phase, 1u << 22);
    }
    // ---- write gradients: thread t owns TMEM lane t of each accumulator.
    if (!bad && !first) {
#pragma unroll 1
        for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + lane_off + kColW3 + c0, v);
            tc::wait_ld();
            for (int i = 0; i < 16; ++i) atomicAdd(grads + kOffW3 + t * kMlpHidden + c0 + i, v[i]);
            tc::tmem_ld16(tmem + lane_off + kColW2 + c0, v);
            tc::wait_ld();
            for (int i = 0; i < 16; ++i) atomicAdd(grads + kOffW2 + t * kMlpHidden + c0 + i, v[i]);
        }
#pragma unroll 1
        for (int c0 = 0; c0 < kMlpIn; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + lane_off + kColW1 + c0, v);
            tc::wait_ld();
            for (int i = 0; i < 16; ++i) atomicAdd(grads + kOffW1 + (c0 + i) * kMlpHidden + t, v[i]);
        }
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (!bad) {
        atomicAdd(grads + kOffB1 + t, db1[t]);
        atomicAdd(grads + kOffB2 + t, db2[t]);
        atomicAdd(grads + kOffB3 + t, db3[t]);
        atomicAdd(grads + kOffW4 + t, dw4[t]);
        if (t == 0) {
            atomicAdd(grads + kOffB4, gv[4 * kMlpHidden]);
            atomicAdd(loss_sum, gv[5 * kMlpHidden + 1]);
        }
    }
    if (warp == 0) tc::tmem_free(tmem, 512);
}

// Adam on the FP32 masters (bias-corrected), then the BF16 images are re-packed.
__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                                float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

cudaError_t mlp_train_grads(const uint16_t* d_x, const uint8_t* d_y, int rows, const uint8_t* d_images,
                            const float* d_params, float* d_grads, float* d_loss, int* d_err, int num_sms,
                            cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_grads, 0, sizeof(float) * kMlpParams, st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(d_loss, 0, sizeof(float), st);
    if (e != cudaSuccess) return e;
    if (rows <= 0) return cudaSuccess;
    e = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem);
    if (e != cudaSuccess) return e;
    const int tiles = (rows + 127) / 128;
    const int grid = tiles < num_sms ? tiles : num_sms;
    mlp_train_kernel<<<grid, 128, kTrainSmem, st>>>(d_x, d_y, rows, reinterpret_cast<const uint4*>(d_images), d_params,
                                                    d_grads, d_loss, d_err);
    return cudaGetLastError();
}

cudaError_t mlp_adam(float* d_params, const float* d_grads, float* d_m, float* d_v, long long step, float lr,
                     cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(d_params, d_grads, d_m, d_v, kMlpParams, lr, b1, b2,
                                                              1e-8f, c1, c2);
    return cudaGetLastError();
}

cudaError_t mlp_pack(const float* d_params, uint8_t* d_images, cudaStream_t st) {
    const int n = kMlpHidden * kMlpIn + 2 * kMlpHidden * kMlpHidden + 3 * kMlpHidden * 16;
    mlp_pack_kernel<<<(n + 255) / 256, 256, 0, st>>>(d_params, d_images);
    return cudaGetLastError();
}

cudaError_t mlp_forward(const uint16_t* d_x, int rows, const uint8_t* d_images, const float* d_params,
                        float* d_logits, int* d_err, int num_sms, cudaStream_t st, const int* d_rows) {
    if (rows <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem);
    if (e != cudaSuccess) return e;
    const int tiles = (rows + 127) / 128;
    const int ctas = (tiles + kFwdGroups - 1) / kFwdGroups;
    const int grid = ctas < num_sms ? ctas : num_sms;
    mlp_forward_kernel<<<grid, 128 * kFwdGroups, kFwdSmem, st>>>(d_x, rows, d_rows,
                                                                 reinterpret_cast<const uint4*>(d_images), d_params,
                                                                 d_logits, d_err);
    return cudaGetLastError();
}

}  // namespace bcc

// ====================================================================== C ABI
namespace {

bcc_status mlp_fail(bcc_ctx* c, bcc_status s, const char* msg) {
    if (c) c->err = msg;
    return s;
}

int sm_count(int dev) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

}  // namespace

extern "C" {

int32_t bcc_mlp_num_params(void) { return bcc::kMlpParams; }

bcc_status bcc_mlp_set_params(bcc_ctx* ctx, const float* params, int32_t n) {
    if (!ctx || !params || n != bcc::kMlpParams) return mlp_fail(ctx, BCC_ERR_INVALID_ARGUMENT, "bad MLP parameters");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return BCC_ERR_CUDA;
    bcc::MlpState& m = ctx->mlp;
    const size_t pb = sizeof(float) * bcc::kMlpParams;
    if (m.params.ensure(pb) != cudaSuccess || m.grads.ensure(pb) != cudaSuccess || m.adam_m.ensure(pb) != cudaSuccess ||
        m.adam_v.ensure(pb) != cudaSuccess || m.images.ensure(bcc::kImagesBytes) != cudaSuccess)
        return mlp_fail(ctx, BCC_ERR_CUDA, "MLP allocation failed");
    if (cudaMemcpy(m.params.p, params, pb, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(m.adam_m.p, 0, pb) != cudaSuccess || cudaMemset(m.adam_v.p, 0, pb) != cudaSuccess)
        return mlp_fail(ctx, BCC_ERR_CUDA, "MLP upload failed");
    if (bcc::mlp_pack(m.params.as<float>(), m.images.as<uint8_t>(), ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return mlp_fail(ctx, BCC_ERR_CUDA, "MLP pack failed");
    m.step = 0;
    m.ready = true;
    return BCC_OK;
}

bcc_status bcc_mlp_get_params(bcc_ctx* ctx, float* params, int32_t n) {
    if (!ctx || !params || n != bcc::kMlpParams || !ctx->mlp.ready) return BCC_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess ||
        cudaMemcpy(params, ctx->mlp.params.p, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return BCC_ERR_CUDA;
    return BCC_OK;
}

bcc_status bcc_mlp_forward(bcc_ctx* ctx, const void* d_x_bf16, int32_t rows, float* d_logits, void* stream) {
    if (!ctx || !ctx->mlp.ready) return mlp_fail(ctx, BCC_ERR_INVALID_ARGUMENT, "MLP parameters not set");
    if (rows < 0 || (rows > 0 && (!d_x_bf16 || !d_logits))) return mlp_fail(ctx, BCC_ERR_INVALID_ARGUMENT, "bad MLP input");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return BCC_ERR_CUDA;
    if (ctx->error_flag.ensure(sizeof(int)) != cudaSuccess) return BCC_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(ctx->error_flag.p, 0, sizeof(int), st) != cudaSuccess) return BCC_ERR_CUDA;
    if (bcc::mlp_forward(static_cast<const uint16_t*>(d_x_bf16), rows, ctx->mlp.images.as<uint8_t>(),
                         ctx->mlp.params.as<float>(), d_logits, ctx->error_flag.as<int>(), sm_count(ctx->device),
                         st) != cudaSuccess)
        return mlp_fail(ctx, BCC_ERR_CUDA, "MLP forward launch failed");
    return BCC_OK;
}

// Gradients (and summed loss) of the mean BCE over `rows` labelled rows,
// computed by the tensor-core training kernel; written to host arrays.
bcc_status bcc_mlp_gradients(bcc_ctx* ctx, const void* d_x_bf16, const uint8_t* d_labels, int32_t rows,
                             float* h_grads, float* h_loss) {
    if (!ctx || !ctx->mlp.ready) return mlp_fail(ctx, BCC_ERR_INVALID_ARGUMENT, "MLP parameters not set");
    if (rows < 0 || (rows > 0 && (!d_x_bf16 || !d_labels))) return BCC_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return BCC_ERR_CUDA;
    bcc::MlpState& m = ctx->mlp;
    if (ctx->error_flag.ensure(sizeof(int)) != cudaSuccess || m.logits.ensure(sizeof(float) * 4) != cudaSuccess)
        return BCC_ERR_CUDA;
    cudaStream_t st = ctx->stream;
    if (cudaMemsetAsync(ctx->error_flag.p, 0, sizeof(int), st) != cudaSuccess) return BCC_ERR_CUDA;
    if (bcc::mlp_train_grads(static_cast<const uint16_t*>(d_x_bf16), d_labels, rows, m.images.as<uint8_t>(),
                             m.params.as<float>(), m.grads.as<float>(), m.logits.as<float>(), ctx->error_flag.as<int>(),
                             sm_count(ctx->device), st) != cudaSuccess)
        return mlp_fail(ctx, BCC_ERR_CUDA, "MLP training kernel launch failed");
    int flag = 0;
    if (cudaMemcpyAsync(&flag, ctx->error_flag.p, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return BCC_ERR_CUDA;
    if (flag) return mlp_fail(ctx, BCC_ERR_TIMEOUT, "MLP training kernel wait timed out");
    if (h_grads && cudaMemcpy(h_grads, m.grads.p, sizeof(float) * bcc::kMlpParams, cudaMemcpyDeviceToHost) != cudaSuccess)
        return BCC_ERR_CUDA;
    if (h_loss && cudaMemcpy(h_loss, m.logits.p, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return BCC_ERR_CUDA;
    return BCC_OK;
}

// One optimisation step: gradients of the batch, Adam update (lr), re-pack.
bcc_status bcc_mlp_train_step(bcc_ctx* ctx, const void* d_x_bf16, const uint8_t* d_labels, int32_t rows, float lr,
                              float* h_loss) {
    bcc_status s = bcc_mlp_gradients(ctx, d_x_bf16, d_labels, rows, nullptr, h_loss);
    if (s != BCC_OK) return s;
    bcc::MlpState& m = ctx->mlp;
    m.step += 1;
    if (bcc::mlp_adam(m.params.as<float>(), m.grads.as<float>(), m.adam_m.as<float>(), m.adam_v.as<float>(), m.step, lr,
                      ctx->stream) != cudaSuccess ||
        bcc::mlp_pack(m.params.as<float>(), m.images.as<uint8_t>(), ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return mlp_fail(ctx, BCC_ERR_CUDA, "MLP update failed");
    return BCC_OK;
}

}  // extern "C"
