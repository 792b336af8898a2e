// bcc_kernels.cu -- sm_100a kernels of the batch edge collision checker.
//
// Pipeline of one check (all on one stream):
//   1. edge_steps_kernel   n per edge (reference discretisation, src/batch_cc.cu:103-107)
//   2. scan_kernel         exclusive prefix sum of 32 n -> per-edge sample offsets
//   3. fk_kernel           one thread per (edge, sample): FK of every robot sphere
//                          into the sample table, env-independent, computed once
//                          instead of once per environment as in the reference
//   4. self_kernel         self-collision of every sample (src/utils.cuh:1192-5440),
//                          OR-reduced per edge; env-independent
//   5. swept_kernel        per (edge, link) AABB of the link's bounding sphere over
//                          all the edge's samples (cull volume)
//   6. check_kernel        CTA = one edge x a tile of environments; each warp takes
//                          one environment at a time: bulk-copies its primitives
//                          into shared memory (cp.async.bulk + mbarrier, double
//                          buffered), culls (primitive, link) pairs against the swept
//                          AABBs, then walks (sample, pair) items 32 at a time in
//                          check order with a warp-ballot exit on the first hit.
#include <cstdint>
#include <cuda_runtime.h>

#include "bcc_device.cuh"
#include "bcc_kernels.h"
#include "robot_panda.h"

namespace bcc {

// ------------------------------------------------------------------ tables
template <class M>
struct DevTables {
    int env_bound[M::num_env_groups];
    int leaf_begin[M::num_env_groups + 1];
    int leaves[M::num_env_leaves];
    int self_bound[M::num_self_groups][2];
    int self_pair_begin[M::num_self_groups + 1];
    unsigned char self_pairs[M::num_self_pairs][2];
    float sphere_radius[M::num_spheres];
};

__constant__ DevTables<PandaModel> c_tab_panda;

template <class M>
__device__ __forceinline__ const DevTables<M>& tab();
template <>
__device__ __forceinline__ const DevTables<PandaModel>& tab<PandaModel>() {
    return c_tab_panda;
}

template <class M>
static DevTables<M> host_tables() {
    DevTables<M> t;
    for (int g = 0; g < M::num_env_groups; ++g) t.env_bound[g] = M::env_bound[g];
    for (int g = 0; g <= M::num_env_groups; ++g) t.leaf_begin[g] = M::env_leaf_begin[g];
    for (int i = 0; i < M::num_env_leaves; ++i) t.leaves[i] = M::env_leaves[i];
    for (int g = 0; g < M::num_self_groups; ++g) {
        t.self_bound[g][0] = M::self_bound[g][0];
        t.self_bound[g][1] = M::self_bound[g][1];
    }
    for (int g = 0; g <= M::num_self_groups; ++g) t.self_pair_begin[g] = M::self_pair_begin[g];
    for (int i = 0; i < M::num_self_pairs; ++i) {
        t.self_pairs[i][0] = M::self_pairs[i][0];
        t.self_pairs[i][1] = M::self_pairs[i][1];
    }
    for (int s = 0; s < M::num_spheres; ++s) t.sphere_radius[s] = M::sphere_radius[s];
    return t;
}

cudaError_t upload_robot_tables(int robot) {
    if (robot != 0) return cudaErrorInvalidValue;
    DevTables<PandaModel> t = host_tables<PandaModel>();
    return cudaMemcpyToSymbol(c_tab_panda, &t, sizeof(t));
}

// ------------------------------------------------------------------ 1. steps
template <class M>
__global__ void edge_steps_kernel(const float* __restrict__ edges, int E, int resolution,
                                  int* __restrict__ steps) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    float s[M::dof], t[M::dof];
#pragma unroll
    for (int j = 0; j < M::dof; ++j) {
        s[j] = edges[(size_t)e * 2 * M::dof + j];
        t[j] = edges[(size_t)e * 2 * M::dof + M::dof + j];
    }
    // Non-finite endpoints would give an unbounded step count: clamp, and let the
    // host reject the resulting sample total (BCC_ERR_LIMIT).
    const int n = edge_steps<M::dof>(s, t, resolution);
    steps[e] = (n < 1 || n > (1 << 20)) ? (1 << 20) : n;
}

// ------------------------------------------------------------------ 2. scan
// Single-CTA exclusive scan of 32*steps[e] into offs[e], offs[E] = total.
__global__ void scan_kernel(const int* __restrict__ steps, int E, int* __restrict__ offs) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < E; base += blockDim.x) {
        const int i = base + threadIdx.x;
        int v = (i < E) ? kLanes * steps[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int w = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const int warp_prefix = warp ? warp_sums[warp - 1] : 0;
        if (i < E) offs[i] = carry + warp_prefix + x - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += warp_prefix + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) offs[E] = carry;
}

// ------------------------------------------------------------------ 3. FK
template <class M, int S>
struct WriteSpheres {
    __device__ __forceinline__ static void run(const Frames<M>& F, float4* __restrict__ out) {
        WriteSpheres<M, S - 1>::run(F, out);
        out[S - 1] = fk_sphere<M, S - 1>(F);
    }
};
template <class M>
struct WriteSpheres<M, 0> {
    __device__ __forceinline__ static void run(const Frames<M>&, float4*) {}
};

// Sample table row: num_spheres float4 (centre xyz, radius), one row per
// (edge, sample) in edge order then sample index order.
template <class M>
__global__ void __launch_bounds__(128) fk_kernel(const float* __restrict__ edges, int E,
                                                 const int* __restrict__ steps,
                                                 const int* __restrict__ offs,
                                                 float4* __restrict__ table,
                                                 int* __restrict__ row_edge) {
    const int total = offs[E];
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= total) return;
    // edge of this row: binary search over offs
    int lo = 0, hi = E - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (offs[mid] <= row) lo = mid; else hi = mid - 1;
    }
    const int e = lo;
    const int k = row - offs[e];
    float s[M::dof], t[M::dof], q[M::dof];
#pragma unroll
    for (int j = 0; j < M::dof; ++j) {
        s[j] = edges[(size_t)e * 2 * M::dof + j];
        t[j] = edges[(size_t)e * 2 * M::dof + M::dof + j];
    }
    edge_sample<M::dof>(s, t, steps[e], k, q);
    Frames<M> F;
    fk_frames<M>(q, F);
    WriteSpheres<M, M::num_spheres>::run(F, table + (size_t)row * M::num_spheres);
    row_edge[row] = e;
}

// ------------------------------------------------------------------ 4. self
__device__ __forceinline__ bool self_hit(float4 a, float4 b) {
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    const float rs = a.w + b.w;
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz)) - rs * rs < 0.0f;
}

template <class M>
__global__ void __launch_bounds__(128) self_kernel(const float4* __restrict__ table, int total,
                                                   const int* __restrict__ row_edge,
                                                   int* __restrict__ edge_self) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= total) return;
    const float4* sp = table + (size_t)row * M::num_spheres;
    const DevTables<M>& T = tab<M>();
    bool hit = false;
    for (int g = 0; g < M::num_self_groups && !hit; ++g) {
        if (!self_hit(sp[T.self_bound[g][0]], sp[T.self_bound[g][1]])) continue;
        for (int k = T.self_pair_begin[g]; k < T.self_pair_begin[g + 1]; ++k) {
            if (self_hit(sp[T.self_pairs[k][0]], sp[T.self_pairs[k][1]])) {
                hit = true;
                break;
            }
        }
    }
    if (hit) atomicOr(edge_self + row_edge[row], 1);
}

// ------------------------------------------------------------------ 5. swept
// One warp per edge: AABB (centre, half-size) of every env group's bounding
// sphere over the edge's samples, inflated by radius + 0.005 + cull margin.
template <class M>
__global__ void swept_kernel(const float4* __restrict__ table, const int* __restrict__ offs, int E,
                             float4* __restrict__ swept) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= E) return;
    const int r0 = offs[warp], r1 = offs[warp + 1];
    const DevTables<M>& T = tab<M>();
    for (int g = 0; g < M::num_env_groups; ++g) {
        const int b = T.env_bound[g];
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int r = r0 + lane; r < r1; r += 32) {
            const float4 c = table[(size_t)r * M::num_spheres + b];
            lo[0] = fminf(lo[0], c.x); lo[1] = fminf(lo[1], c.y); lo[2] = fminf(lo[2], c.z);
            hi[0] = fmaxf(hi[0], c.x); hi[1] = fmaxf(hi[1], c.y); hi[2] = fmaxf(hi[2], c.z);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
                hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
            }
        }
        if (lane == 0) {
            const float pad = T.sphere_radius[b] + kEnvInflate + kCullMargin;
            float4 c, h;
            c.x = 0.5f * (lo[0] + hi[0]); c.y = 0.5f * (lo[1] + hi[1]); c.z = 0.5f * (lo[2] + hi[2]);
            h.x = 0.5f * (hi[0] - lo[0]) + pad; h.y = 0.5f * (hi[1] - lo[1]) + pad;
            h.z = 0.5f * (hi[2] - lo[2]) + pad;
            c.w = 0.0f; h.w = 0.0f;
            swept[((size_t)warp * M::num_env_groups + g) * 2 + 0] = c;
            swept[((size_t)warp * M::num_env_groups + g) * 2 + 1] = h;
        }
    }
}

// ------------------------------------------------------------------ 6. check
struct CheckSmemLayout {
    int max_prims;  // per environment, rounded up
    __host__ __device__ size_t prim_bytes() const { return (size_t)max_prims * kPrimF4 * 16; }
    __host__ __device__ size_t pair_bytes() const { return (((size_t)max_prims * 16 * 2) + 15) & ~(size_t)15; }
    __host__ __device__ size_t per_warp() const { return 2 * prim_bytes() + pair_bytes(); }
};

template <class M, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) check_kernel(CheckParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bars[WARPS][2];
    __shared__ float4 s_swept[M::num_env_groups][2];

    const int e = blockIdx.y;
    const int tile0 = blockIdx.x * P.envs_per_cta;
    const int tile1 = min(tile0 + P.envs_per_cta, P.num_envs);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // Self-colliding edge: every environment's verdict is "collision".
    if (P.edge_self[e]) {
        for (int v = tile0 + threadIdx.x; v < tile1; v += blockDim.x)
            P.results[(size_t)e * P.num_envs + v] = 1;
        return;
    }
    if (threadIdx.x < M::num_env_groups * 2)
        (&s_swept[0][0])[threadIdx.x] = P.swept[(size_t)e * M::num_env_groups * 2 + threadIdx.x];
    if (lane == 0) {
        mbar_init(&bars[warp][0], 1);
        mbar_init(&bars[warp][1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const CheckSmemLayout L{P.max_prims};
    unsigned char* wbase = smem + (size_t)warp * L.per_warp();
    float4* pbuf[2] = {reinterpret_cast<float4*>(wbase), reinterpret_cast<float4*>(wbase + L.prim_bytes())};
    uint16_t* pairs = reinterpret_cast<uint16_t*>(wbase + 2 * L.prim_bytes());

    const int n = P.steps[e];
    const int S = kLanes * n;
    const size_t row0 = (size_t)P.offs[e];
    const DevTables<M>& T = tab<M>();

    // Per-buffer mbarrier phase; pending = a bulk copy was issued and not yet waited on.
    uint32_t phase[2] = {0u, 0u};
    bool pending[2] = {false, false};
    int v = tile0 + warp;
    auto issue = [&](int env, int b) {
        const int p0 = P.env_off[env], p1 = P.env_off[env + 1];
        const uint32_t bytes = (uint32_t)(p1 - p0) * kPrimF4 * 16u;
        if (bytes) {
            if (lane == 0) bulk_copy_g2s(pbuf[b], P.prims + (size_t)p0 * kPrimF4, bytes, &bars[warp][b]);
            pending[b] = true;
        }
    };
    if (v < tile1) issue(v, 0);
    int buf = 0;
    bool failed = false;
    for (; v < tile1; v += WARPS, buf ^= 1) {
        const int nv = v + WARPS;
        __syncwarp();
        if (nv < tile1) issue(nv, buf ^ 1);
        if (pending[buf]) {
            if (!mbar_wait_bounded(&bars[warp][buf], phase[buf], 1u << 22)) {
                failed = true;
                break;
            }
            phase[buf] ^= 1u;
            pending[buf] = false;
        }
        const int np = P.env_off[v + 1] - P.env_off[v];
        const float4* prim = pbuf[buf];

        // Cull: (primitive, link) pairs whose AABBs overlap; compact into `pairs`.
        int C = 0;
        for (int p0 = 0; p0 < np; p0 += 32) {
            const int p = p0 + lane;
            uint32_t mask = 0;
            if (p < np) {
                const float4 c = prim[p * kPrimF4 + 0];
                const float4 h = prim[p * kPrimF4 + 4];
#pragma unroll
                for (int g = 0; g < M::num_env_groups; ++g) {
                    const float4 sc = s_swept[g][0], sh = s_swept[g][1];
                    const bool ov = fabsf(c.x - sc.x) <= h.x + sh.x && fabsf(c.y - sc.y) <= h.y + sh.y &&
                                    fabsf(c.z - sc.z) <= h.z + sh.z;
                    mask |= (uint32_t)ov << g;
                }
            }
            const int cnt = __popc(mask);
            int x = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            int w = C + x - cnt;
            while (mask) {
                const int g = __ffs(mask) - 1;
                mask &= mask - 1;
                pairs[w++] = (uint16_t)((p << 4) | g);
            }
            C += __shfl_sync(0xffffffffu, x, 31);
        }
        __syncwarp();

        // Walk (sample rank, pair) items, 32 per step, in check order.
        bool collide = false;
        if (C > 0) {
            const int total = S * C;
            const int dr = 32 / C, dc = 32 % C;
            int r = lane / C, c = lane - (lane / C) * C;
            for (int w0 = 0; w0 < total; w0 += 32) {
                bool hit = false;
                if (w0 + lane < total) {
                    const int k = reference_rank_to_sample(r, n);
                    const uint32_t pr = pairs[c];
                    const int p = (int)(pr >> 4), g = (int)(pr & 15u);
                    const float4* rec = prim + p * kPrimF4;
                    const float4* row = P.table + (row0 + (size_t)k) * M::num_spheres;
                    float4 bs = row[T.env_bound[g]];
                    bs.w += kEnvInflate;
                    if (sphere_hits_prim(bs, rec)) {
                        for (int li = T.leaf_begin[g]; li < T.leaf_begin[g + 1]; ++li) {
                            float4 ls = row[T.leaves[li]];
                            ls.w += kEnvInflate;
                            if (sphere_hits_prim(ls, rec)) {
                                hit = true;
                                break;
                            }
                        }
                    }
                }
                if (__any_sync(0xffffffffu, hit)) {
                    collide = true;
                    break;
                }
                c += dc;
                r += dr;
                if (c >= C) {
                    c -= C;
                    ++r;
                }
            }
        }
        if (lane == 0) P.results[(size_t)e * P.num_envs + v] = collide ? 1 : 0;
    }
    if (failed) {
        if (lane == 0) atomicOr(P.error_flag, 1);
        // Do not leave with a bulk copy still writing this CTA's shared memory.
        for (int b = 0; b < 2; ++b)
            if (pending[b]) mbar_wait_bounded(&bars[warp][b], phase[b], 1u << 22);
    }
}

// ------------------------------------------------------------------ launchers
size_t check_smem_bytes(int max_prims, int warps) {
    CheckSmemLayout L{max_prims};
    return L.per_warp() * warps;
}

template <class M>
static cudaError_t run_steps(const PipelineArgs& a, cudaStream_t st) {
    const int E = a.num_edges;
    if (a.stage_events) cudaEventRecord(a.stage_events[0], st);
    edge_steps_kernel<M><<<(E + 255) / 256, 256, 0, st>>>(a.d_edges, E, a.resolution, a.steps);
    scan_kernel<<<1, 1024, 0, st>>>(a.steps, E, a.offs);
    return cudaGetLastError();
}

template <class M, int W>
static cudaError_t launch_check_w(const CheckParams& P, int E, cudaStream_t st) {
    const size_t smem = check_smem_bytes(P.max_prims, W);
    cudaError_t err = cudaFuncSetAttribute(check_kernel<M, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
    if (err != cudaSuccess) return err;
    dim3 grid((P.num_envs + P.envs_per_cta - 1) / P.envs_per_cta, E);
    check_kernel<M, W><<<grid, W * 32, smem, st>>>(P);
    return cudaGetLastError();
}

template <class M>
static cudaError_t run_check(const PipelineArgs& a, cudaStream_t st) {
    const int E = a.num_edges;
    const int R = a.total_rows;
    cudaEvent_t* ev = a.stage_events;
    if (ev) cudaEventRecord(ev[1], st);
    if (R > 0) {
        fk_kernel<M><<<(R + 127) / 128, 128, 0, st>>>(a.d_edges, E, a.steps, a.offs, a.table, a.row_edge);
    }
    if (ev) cudaEventRecord(ev[2], st);
    cudaError_t err = cudaMemsetAsync(a.edge_self, 0, sizeof(int) * E, st);
    if (err != cudaSuccess) return err;
    if (R > 0) self_kernel<M><<<(R + 127) / 128, 128, 0, st>>>(a.table, R, a.row_edge, a.edge_self);
    if (ev) cudaEventRecord(ev[3], st);
    swept_kernel<M><<<(E * 32 + 255) / 256, 256, 0, st>>>(a.table, a.offs, E, a.swept);
    if (ev) cudaEventRecord(ev[4], st);

    CheckParams P;
    P.prims = a.prims;
    P.env_off = a.env_off;
    P.num_envs = a.num_envs;
    P.max_prims = a.max_prims;
    P.envs_per_cta = a.envs_per_cta;
    P.steps = a.steps;
    P.offs = a.offs;
    P.table = a.table;
    P.swept = a.swept;
    P.edge_self = a.edge_self;
    P.results = a.d_results;
    P.error_flag = a.error_flag;
    switch (a.warps) {
        case 8: err = launch_check_w<M, 8>(P, E, st); break;
        case 4: err = launch_check_w<M, 4>(P, E, st); break;
        case 2: err = launch_check_w<M, 2>(P, E, st); break;
        case 1: err = launch_check_w<M, 1>(P, E, st); break;
        default: return cudaErrorInvalidValue;
    }
    if (ev) cudaEventRecord(ev[5], st);
    return err;
}

cudaError_t launch_steps(int robot, const PipelineArgs& a, cudaStream_t st) {
    if (robot != 0) return cudaErrorInvalidValue;
    return run_steps<PandaModel>(a, st);
}

cudaError_t launch_check(int robot, const PipelineArgs& a, cudaStream_t st) {
    if (robot != 0) return cudaErrorInvalidValue;
    return run_check<PandaModel>(a, st);
}

int robot_num_spheres(int robot) { return robot == 0 ? PandaModel::num_spheres : -1; }
int robot_num_env_groups(int robot) { return robot == 0 ? PandaModel::num_env_groups : -1; }
int robot_dof(int robot) { return robot == 0 ? PandaModel::dof : -1; }

}  // namespace bcc
