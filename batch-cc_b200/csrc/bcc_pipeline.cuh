// bcc_pipeline.cuh -- robot-templated kernels and launchers of the batch edge
// collision checker (sm_100a).
//
// Included by exactly one translation unit per robot (bcc_robot_<name>.cu),
// which defines the robot's __constant__ tables, specialises tab<Model>() to
// return them and instantiates everything below for its model through
// robot_ops_of<Model>().
//
// Pipeline of one check (all on one stream):
//   1. edge_steps_kernel   n per edge (reference discretisation, src/batch_cc.cu:103-107)
//   2. scan_kernel         exclusive prefix sum of 32 n -> per-edge sample offsets
//   3. fk_kernel           one thread per (edge, sample): FK of every robot sphere
//                          into the sample table, env-independent, computed once
//                          instead of once per environment as in the reference
//   4. self_kernel         self-collision of every sample (src/utils.cuh:1192-5440
//                          for Panda), OR-reduced per edge; env-independent
//   5. swept_kernel        per (edge, link) AABB of the link's cull sphere over
//                          all the edge's samples
//   6. check_kernel        CTA = one environment x a tile of edges.  The
//                          environment's primitive records are staged into shared
//                          memory once by a cp.async.bulk copy and reused by every
//                          edge of the tile.  Each warp takes one edge at a time:
//                          lane g turns link g's swept AABB into three slab ranges
//                          and ANDs three 64-bit primitive masks of the
//                          environment's interval-mask tables (the cull, read
//                          through L1), the surviving (primitive, link) pairs are
//                          compacted (lane g writes link g's), and the warp walks
//                          (sample, pair) items 32 at a time in check order with a
//                          warp-ballot exit on the first hit.
//
// Gate semantics.  The reference tests a link's leaves only after the link's
// bounding sphere hit SOME primitive (fkcc: `if (bound in collision) { if
// (leaf in collision) return false; ... }`).  Per (sample, primitive, link)
// item the checker tests the bound against that primitive and, on a hit, every
// leaf against it.  That is the same verdict wherever the leaves lie inside
// the bound.  For the leaves that stick out of their bound (Fetch, Baxter:
// up to 0.6 mm, the model's env_over_count / env_cull_pad) the checker also
// tests them against primitives the bound misses but the padded bound reaches,
// and a hit there counts only after a scan of the whole environment confirms
// that the bound hits some primitive at that sample.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include <cuda_bf16.h>

#include "bcc_device.cuh"
#include "bcc_kernels.h"
#include "bcc_mlp.h"

namespace bcc {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------ tables
template <class M>
struct DevTables {
    int env_bound[M::num_env_groups];
    int leaf_begin[M::num_env_groups + 1];
    int over_count[M::num_env_groups];
    float cull_pad[M::num_env_groups];
    // Certain-hit radius of env group g (0: none): a primitive whose core lies
    // within rho + cert_r[g] of the bound's centre is hit by a leaf of g.
    float cert_r[M::num_env_groups];
    int self_bound[M::num_self_groups][2];
    int self_pair_begin[M::num_self_groups + 1];
    unsigned char self_pairs[M::num_self_pairs][2];
    // Self groups whose leaf pairs are every leaf of side 0 against every leaf
    // of side 1 (self_prod[g] = 1; at most 32 leaves a side, each side's leaves
    // rigid with its bound): the sides' leaves (row positions) and, per side,
    // how far its leaves may reach outside its bound plus a margin for FP32
    // rounding.  A leaf that misses the other side's bound grown by that side's
    // pad misses every leaf of that side.
    unsigned char self_prod[M::num_self_groups];
    int self_la_begin[M::num_self_groups + 1], self_lb_begin[M::num_self_groups + 1];
    unsigned char self_la[M::num_self_pairs], self_lb[M::num_self_pairs];
    float self_pad[M::num_self_groups][2];
    float sphere_radius[M::num_spheres];  // by sample-table position
    float s_m[M::dof], s_a[M::dof];       // joint-limit scale q = u * s_m + s_a
};

// Specialised by the robot's translation unit to return its __constant__ tables.
template <class M>
__device__ __forceinline__ const DevTables<M>& tab();

// Margin (m) added to a side's containment excess in the self groups' leaf
// filter: far above the FP32 rounding of FK-computed centres (~1e-6 m).
constexpr double kSelfFilterMargin = 1e-4;

// Certain-hit radius of an environment group.  Leaf l (rigid with the bound's
// frame, centre c_l, radius r_l) hits a primitive when the distance from c_l
// to the primitive's core is below r_l + kEnvInflate + rho, and that distance
// is at most the bound centre's distance d_b plus |c_l - c_b| (distance to a
// convex set is 1-Lipschitz).  So d_b < rho + max_l (r_l + kEnvInflate -
// |c_l - c_b|) proves a leaf hit: the leaf penetrates by more than the margin
// subtracted here, far above FP32 rounding of FK-computed centres, so the
// reference's own leaf test (src/utils.cuh:806-1190) finds that hit too.
constexpr double kCertMargin = 1e-4;

template <class M>
float cert_radius(int g) {
    const int b = M::env_bound[g];
    double best = 0.0;
    for (int k = M::env_leaf_begin[g]; k < M::env_leaf_begin[g + 1]; ++k) {
        const int l = M::env_leaves[k];
        if (M::sphere_frame[l] != M::sphere_frame[b]) continue;  // not rigid with the bound
        // r_l <= r_b keeps the radius within r_b + kEnvInflate, so a certain hit
        // is also a bound hit (the reference tests leaves only after one)
        if (M::sphere_radius[l] > M::sphere_radius[b]) continue;
        double d2 = 0.0;
        for (int c = 0; c < 3; ++c) {
            const double d = M::sphere_local[l][c] - M::sphere_local[b][c];
            d2 += d * d;
        }
        const double v = (double)M::sphere_radius[l] + (double)kEnvInflate - std::sqrt(d2) - kCertMargin;
        best = v > best ? v : best;
    }
    // rounded down to float: the test stays conservative
    float f = (float)best;
    if ((double)f > best) f = std::nextafter(f, 0.0f);
    return f;
}

template <class M>
void self_products(DevTables<M>& t) {
    int na_tot = 0, nb_tot = 0;
    for (int g = 0; g < M::num_self_groups; ++g) {
        const int k0 = M::self_pair_begin[g], k1 = M::self_pair_begin[g + 1];
        int la[M::num_spheres], lb[M::num_spheres], na = 0, nb = 0;
        bool in_a[M::num_spheres] = {}, in_b[M::num_spheres] = {};
        for (int k = k0; k < k1; ++k) {
            const int a = M::self_pairs[k][0], b = M::self_pairs[k][1];
            if (!in_a[a]) { in_a[a] = true; la[na++] = a; }
            if (!in_b[b]) { in_b[b] = true; lb[nb++] = b; }
        }
        // a product: as many distinct pairs as |A| x |B| (each pair is in A x B)
        bool prod = na <= 32 && nb <= 32 && na * nb == k1 - k0;
        for (int k = k0; k < k1 && prod; ++k)
            for (int k2 = k0; k2 < k; ++k2)
                if (M::self_pairs[k2][0] == M::self_pairs[k][0] && M::self_pairs[k2][1] == M::self_pairs[k][1])
                    prod = false;
        for (int side = 0; side < 2 && prod; ++side) {
            const int b = M::self_bound[g][side];
            double excess = 0.0;
            for (int i = 0; i < (side ? nb : na); ++i) {
                const int l = side ? lb[i] : la[i];
                if (M::sphere_frame[l] != M::sphere_frame[b]) { prod = false; break; }
                double d2 = 0.0;
                for (int c = 0; c < 3; ++c) {
                    const double d = M::sphere_local[l][c] - M::sphere_local[b][c];
                    d2 += d * d;
                }
                const double ex = std::sqrt(d2) + M::sphere_radius[l] - M::sphere_radius[b];
                excess = ex > excess ? ex : excess;
            }
            t.self_pad[g][side] = (float)(excess + kSelfFilterMargin);
        }
        t.self_prod[g] = prod ? 1 : 0;
        t.self_la_begin[g] = na_tot;
        t.self_lb_begin[g] = nb_tot;
        if (prod) {
            for (int i = 0; i < na; ++i) t.self_la[na_tot++] = (unsigned char)M::table_pos[la[i]];
            for (int i = 0; i < nb; ++i) t.self_lb[nb_tot++] = (unsigned char)M::table_pos[lb[i]];
        } else {
            t.self_pad[g][0] = t.self_pad[g][1] = 0.0f;
        }
    }
    t.self_la_begin[M::num_self_groups] = na_tot;
    t.self_lb_begin[M::num_self_groups] = nb_tot;
}

template <class M>
DevTables<M> host_tables() {
    static_assert(M::num_env_groups <= kMaxEnvGroups, "one cull lane per link group");
    static_assert(M::num_spheres <= kMaxTableSpheres, "sample-table row width");
    static_assert(M::num_spheres <= 256, "self pairs hold 8-bit row positions");
    static_assert(M::table_tile >= 1 && kMaxTableTile % M::table_tile == 0, "table tiles divide the row padding");
    DevTables<M> t;
    for (int g = 0; g < M::num_env_groups; ++g) {
        t.env_bound[g] = M::env_bound[g];
        t.over_count[g] = M::env_over_count[g];
        t.cull_pad[g] = M::env_cull_pad[g];
        t.cert_r[g] = cert_radius<M>(g);
    }
    for (int g = 0; g <= M::num_env_groups; ++g) t.leaf_begin[g] = M::env_leaf_begin[g];
    // Self tables hold sample-table row positions, not sphere indices.
    for (int g = 0; g < M::num_self_groups; ++g) {
        t.self_bound[g][0] = M::table_pos[M::self_bound[g][0]];
        t.self_bound[g][1] = M::table_pos[M::self_bound[g][1]];
    }
    for (int g = 0; g <= M::num_self_groups; ++g) t.self_pair_begin[g] = M::self_pair_begin[g];
    for (int i = 0; i < M::num_self_pairs; ++i) {
        t.self_pairs[i][0] = (unsigned char)M::table_pos[M::self_pairs[i][0]];
        t.self_pairs[i][1] = (unsigned char)M::table_pos[M::self_pairs[i][1]];
    }
    self_products<M>(t);
    for (int s = 0; s < M::num_spheres; ++s) t.sphere_radius[M::table_pos[s]] = M::sphere_radius[s];
    for (int j = 0; j < M::dof; ++j) {
        t.s_m[j] = M::s_m[j];
        t.s_a[j] = M::s_a[j];
    }
    return t;
}

// Bits of the link-group index in a packed (primitive, group) pair.
template <class M>
constexpr int group_bits() {
    return M::num_env_groups <= 16 ? 4 : 5;
}

// Largest primitive count per environment the 16-bit pair packing allows.
template <class M>
constexpr int max_prims_of() {
    return (1 << (16 - group_bits<M>())) - 1;
}

template <class M>
constexpr bool has_overhang() {
    for (int g = 0; g < M::num_env_groups; ++g)
        if (M::env_over_count[g] > 0) return true;
    return false;
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

// ------------------------------------------------------------------ 3. FK
// Sample table row: num_spheres float4 (centre xyz, radius) in table_pos order
// (env-group bounds, then env leaves, then the rest), one row per (edge,
// sample) in edge order then sample index order; stored in tiles of
// M::table_tile rows (table_index).
// Sample at table position k of edge e: k itself, or with a block
// permutation (inline learned order, one cluster) lane block perm[e][k / n]'s
// sample of the same round, so the reference walk over the table visits the
// samples in learned order.
__device__ __forceinline__ int table_sample(const uint8_t* __restrict__ perm, int e, int n, int k) {
    if (!perm) return k;
    const int blk = k / n;
    return (int)perm[(size_t)e * kLanes + blk] * n + (k - blk * n);
}

template <class M>
__global__ void __launch_bounds__(128) fk_kernel(const float* __restrict__ edges, int E,
                                                 const int* __restrict__ steps,
                                                 const int* __restrict__ offs,
                                                 float4* __restrict__ table,
                                                 int* __restrict__ row_edge, const uint8_t* __restrict__ perm) {
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
    edge_sample<M::dof>(s, t, steps[e], table_sample(perm, e, steps[e], k), q);
    fk_spheres<M>(q, table + table_index<M>(row, 0));
    row_edge[row] = e;
}

__device__ __forceinline__ bool self_hit(float4 a, float4 b) {
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    const float rs = a.w + b.w;
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz)) - rs * rs < 0.0f;
}

__device__ __forceinline__ bool self_hit_pad(float4 a, float4 b, float pad) {
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    const float rs = a.w + b.w + pad;
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz)) - rs * rs < 0.0f;
}

// Self-collision of a warp's rows, one lane per row (sphere s at my[s]; live:
// the lane holds a row), all rows of one edge: group g gates on its bound pair
// and its leaf pairs count only where the gate hit (the reference's
// gate-then-leaves).  The warp walks the groups together, so every table index
// is warp-uniform (constant-cache broadcasts), skips a group's leaves when no
// lane's gate hit, and stops at the first hit in any lane.  A group whose
// leaf pairs are a product of two leaf sets (self_prod) first drops the leaves
// of either side that miss the other side's padded bound -- a leaf of side A
// that misses bound B (grown by B's containment pad) misses every leaf inside
// B -- and tests only the pairs of surviving leaves, skipping those no lane
// keeps; the verdict is the one the full pair list gives.  Warp-uniform.
template <class M>
__device__ __forceinline__ bool self_rows_hit(const float4* my, bool live) {
    const DevTables<M>& T = tab<M>();
    for (int g = 0; g < M::num_self_groups; ++g) {
        const float4 ba = my[T.self_bound[g][0]], bb = my[T.self_bound[g][1]];
        const bool gate = live && self_hit(ba, bb);
        if (!__any_sync(kFull, gate)) continue;
        bool h = false;
        if (T.self_prod[g]) {
            const int a0 = T.self_la_begin[g], na = T.self_la_begin[g + 1] - a0;
            const int b0 = T.self_lb_begin[g], nb = T.self_lb_begin[g + 1] - b0;
            const float pa = T.self_pad[g][0], pb = T.self_pad[g][1];
            uint32_t ma = 0u, mb = 0u;
            for (int i = 0; i < na; ++i) ma |= (uint32_t)self_hit_pad(my[T.self_la[a0 + i]], bb, pb) << i;
            for (int j = 0; j < nb; ++j) mb |= (uint32_t)self_hit_pad(my[T.self_lb[b0 + j]], ba, pa) << j;
            if (!gate || !mb) ma = 0u;
            uint32_t ia = __reduce_or_sync(kFull, ma);
            while (ia) {
                const int i = __ffs(ia) - 1;
                ia &= ia - 1u;
                const uint32_t mj = ((ma >> i) & 1u) ? mb : 0u;
                uint32_t jb = __reduce_or_sync(kFull, mj);
                const float4 la = my[T.self_la[a0 + i]];
                while (jb) {
                    const int j = __ffs(jb) - 1;
                    jb &= jb - 1u;
                    h |= ((mj >> j) & 1u) && self_hit(la, my[T.self_lb[b0 + j]]);
                }
            }
        } else {
            const int k1 = T.self_pair_begin[g + 1];
#pragma unroll 4
            for (int k = T.self_pair_begin[g]; k < k1; ++k)
                h |= self_hit(my[T.self_pairs[k][0]], my[T.self_pairs[k][1]]);
        }
        if (__any_sync(kFull, gate && h)) return true;
    }
    return false;
}

// Row-major tables (tile 1): a thread's row is 16 * num_spheres contiguous
// bytes, so per-thread stores would touch 32 rows per warp instruction.  One
// warp per CTA computes 32 rows into shared memory (odd float4 row stride,
// conflict-free) and then copies the 32 consecutive rows out as one contiguous
// block, 512 bytes per warp store.  While the rows are still in shared memory
// the warp also runs their self-collision check, one lane per row, so the rows
// are never read back from global memory for it.  A block's 32 rows belong to
// one edge (every edge has 32 n rows and starts on a multiple of 32), so the
// first hit in any lane decides the block.  The CTA strides over 32-row blocks.
template <class M>
__global__ void __launch_bounds__(32) fk_staged_kernel(const float* __restrict__ edges, int E,
                                                       const int* __restrict__ steps,
                                                       const int* __restrict__ offs,
                                                       float4* __restrict__ table,
                                                       int* __restrict__ row_edge, const uint8_t* __restrict__ perm,
                                                       int* __restrict__ edge_self) {
    static_assert(M::table_tile == 1, "row-major tables only");
    constexpr int NS = M::num_spheres;
    constexpr int STRIDE = NS | 1;
    extern __shared__ float4 srow[];  // [32][STRIDE]
    const int lane = threadIdx.x;
    const int total = offs[E];
    for (int base = blockIdx.x * 32; base < total; base += gridDim.x * 32) {
        const int row = base + lane;
        // the block's edge: the last e with offs[e] <= base (one search per block)
        int lo = 0, hi = E - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (offs[mid] <= base) lo = mid; else hi = mid - 1;
        }
        const int e = lo;
        const int n = steps[e];
        if (row < total) {
            float s[M::dof], t[M::dof], q[M::dof];
#pragma unroll
            for (int j = 0; j < M::dof; ++j) {
                s[j] = edges[(size_t)e * 2 * M::dof + j];
                t[j] = edges[(size_t)e * 2 * M::dof + M::dof + j];
            }
            edge_sample<M::dof>(s, t, n, table_sample(perm, e, n, row - offs[e]), q);
            fk_spheres<M>(q, srow + lane * STRIDE);
            row_edge[row] = e;
        }
        __syncwarp();
        const int rows = min(32, total - base);
        const int cnt = rows * NS;
        float4* __restrict__ dst = table + (size_t)base * NS;
        for (int i = lane; i < cnt; i += 32) {
            const int r = i / NS;
            dst[i] = srow[r * STRIDE + (i - r * NS)];
        }
        // self-collision of the block's rows (any hit marks the edge); skipped
        // when another block of the edge has already marked it
        int decided = lane == 0 ? *(volatile const int*)(edge_self + e) : 0;
        if (!__shfl_sync(kFull, decided, 0) && self_rows_hit<M>(srow + lane * STRIDE, row < total) && lane == 0)
            atomicOr(edge_self + e, 1);
        __syncwarp();  // the next block overwrites srow
    }
}

// ------------------------------------------------------------------ 4. self

// Self-collision of one sample row, by one warp (sphere s at sp[s * stride]).
// Lanes test the self groups' bound pairs 32 at a time; the leaf pairs of
// every group whose bound pair hit are then tested 32 at a time (the
// reference's gate-then-leaves, any hit = self-collision).  The tables are in
// shared memory: lanes read different entries, which constant memory would
// serialise.  Warp-uniform result.
template <class M>
__device__ __forceinline__ bool self_row_hits(const float4* sp, const short (*bound)[2], const short* begin,
                                              const unsigned char (*pairs)[2], int stride) {
    constexpr int NG = M::num_self_groups;
    const int lane = threadIdx.x & 31;
    bool hit = false;
    for (int g0 = 0; g0 < NG && !hit; g0 += 32) {
        const int g = g0 + lane;
        const bool gate = g < NG && self_hit(sp[bound[g][0] * stride], sp[bound[g][1] * stride]);
        uint32_t gm = __ballot_sync(kFull, gate);
        while (gm && !hit) {
            const int gg = g0 + __ffs(gm) - 1;
            gm &= gm - 1u;
            const int end = begin[gg + 1];
            for (int k0 = begin[gg]; k0 < end && !hit; k0 += 32) {  // warp-uniform trip count
                const int k = k0 + lane;
                const bool h = k < end && self_hit(sp[pairs[k][0] * stride], sp[pairs[k][1] * stride]);
                hit = __any_sync(kFull, h);
            }
        }
    }
    return hit;
}

// One warp per sample row (robots with tiled tables; row-major tables are
// checked inside fk_staged_kernel), rows strided over the grid, each row by
// self_row_hits.  Rows of an edge already known to self-collide are skipped.
constexpr int kSelfThreads = 256;

template <class M>
__global__ void __launch_bounds__(kSelfThreads) self_kernel(const float4* __restrict__ table, int total,
                                                             const int* __restrict__ row_edge,
                                                             int* __restrict__ edge_self) {
    constexpr int NG = M::num_self_groups;
    constexpr int NP = M::num_self_pairs;
    __shared__ short s_bound[NG][2];
    __shared__ short s_begin[NG + 1];
    __shared__ unsigned char s_pairs[NP][2];
    const DevTables<M>& T = tab<M>();
    for (int i = threadIdx.x; i < NG; i += blockDim.x) {
        s_bound[i][0] = (short)T.self_bound[i][0];
        s_bound[i][1] = (short)T.self_bound[i][1];
    }
    for (int i = threadIdx.x; i <= NG; i += blockDim.x) s_begin[i] = (short)T.self_pair_begin[i];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) {
        s_pairs[i][0] = T.self_pairs[i][0];
        s_pairs[i][1] = T.self_pairs[i][1];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < total; row += warps) {
        const int e = row_edge[row];
        int decided = lane == 0 ? *(volatile const int*)(edge_self + e) : 0;
        if (__shfl_sync(kFull, decided, 0)) continue;  // another row already found a self-collision
        const float4* sp = table + table_index<M>(row, 0);  // sphere s at sp[s * M::table_tile]
        const bool hit = self_row_hits<M>(sp, s_bound, s_begin, s_pairs, M::table_tile);
        if (hit && lane == 0) atomicOr(edge_self + e, 1);
    }
}

// ------------------------------------------------------------------ 5. swept
// Slab of x on one axis: the largest s in [0, kGridSlabs) with b[s] <= x (0
// below b[0]); b holds the axis' kGridSlabs + 1 increasing boundaries.
__device__ __forceinline__ int slab_of(const float* __restrict__ b, float x) {
    int s = 0;
#pragma unroll
    for (int step = kGridSlabs / 2; step; step >>= 1)
        if (b[s + step] <= x) s += step;
    return s;
}

// Slab index range of [lo, hi] on one axis of the environment set's cull grid,
// as a triangular table index; -1 when the interval misses every primitive.
__device__ __forceinline__ int slab_tri(float lo, float hi, const float* __restrict__ b) {
    if (!(hi >= b[0]) || !(lo < b[kGridSlabs])) return -1;
    return tri_index(slab_of(b, lo), slab_of(b, hi));
}

// One warp per edge: AABB (lo, hi) of every link group's bounding sphere over
// the edge's samples, inflated by radius + 0.005 + the group's leaf overhang +
// cull margin; and (edge_tri non-null) its slab ranges on the set's cull grid,
// packed tx | ty << 10 | tz << 20 (-1 when some axis misses every primitive).
// Lane g ends up holding group g's box.  Row-major tables: lane g scans group
// g's bound down the rows (a row's bounds are contiguous).  Tiled tables: the
// lanes scan 32 rows of one group at a time (contiguous in a tile) and a
// butterfly reduction hands the box to lane g.
template <class M>
__global__ void swept_kernel(const float4* __restrict__ table, const int* __restrict__ offs, int E,
                             float4* __restrict__ swept, int* __restrict__ edge_tri,
                             const float* __restrict__ bounds) {
    constexpr int G = M::num_env_groups;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= E) return;
    const int r0 = offs[warp], r1 = offs[warp + 1];
    const DevTables<M>& T = tab<M>();
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if constexpr (M::table_tile == 1) {
        // 32 / G row streams: lane s G + g scans group g's bound on rows
        // r0 + s, r0 + s + 32 / G, ... (bounds lead every table row); lane g then
        // folds in the other streams' boxes.
        constexpr int RS = kLanes / G;
        const int rs = lane / G, gl = lane - rs * G;
        if (rs < RS) {
            for (int r = r0 + rs; r < r1; r += RS) {
                const float4 c = table[table_index<M>(r, gl)];
                lo[0] = fminf(lo[0], c.x); lo[1] = fminf(lo[1], c.y); lo[2] = fminf(lo[2], c.z);
                hi[0] = fmaxf(hi[0], c.x); hi[1] = fmaxf(hi[1], c.y); hi[2] = fmaxf(hi[2], c.z);
            }
        }
#pragma unroll
        for (int t = 1; t < RS; ++t) {
            const int src = min(lane + t * G, kLanes - 1);  // lanes >= G read a valid lane and discard it
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                lo[a] = fminf(lo[a], __shfl_sync(kFull, lo[a], src));
                hi[a] = fmaxf(hi[a], __shfl_sync(kFull, hi[a], src));
            }
        }
    } else {
        for (int g = 0; g < G; ++g) {
            float l3[3] = {INFINITY, INFINITY, INFINITY}, h3[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int r = r0 + lane; r < r1; r += 32) {
                const float4 c = table[table_index<M>(r, g)];
                l3[0] = fminf(l3[0], c.x); l3[1] = fminf(l3[1], c.y); l3[2] = fminf(l3[2], c.z);
                h3[0] = fmaxf(h3[0], c.x); h3[1] = fmaxf(h3[1], c.y); h3[2] = fmaxf(h3[2], c.z);
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    l3[a] = fminf(l3[a], __shfl_xor_sync(kFull, l3[a], o));
                    h3[a] = fmaxf(h3[a], __shfl_xor_sync(kFull, h3[a], o));
                }
            }
            if (lane == g) {
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    lo[a] = l3[a];
                    hi[a] = h3[a];
                }
            }
        }
    }
    if (lane >= G) return;
    const int g = lane;
    const float pad = T.sphere_radius[g] + kEnvInflate + T.cull_pad[g] + kCullMargin;
    const float4 l = make_float4(lo[0] - pad, lo[1] - pad, lo[2] - pad, 0.0f);
    const float4 h = make_float4(hi[0] + pad, hi[1] + pad, hi[2] + pad, 0.0f);
    swept[((size_t)warp * G + g) * 2 + 0] = l;
    swept[((size_t)warp * G + g) * 2 + 1] = h;
    if (edge_tri) {
        const int tx = slab_tri(l.x, h.x, bounds);
        const int ty = slab_tri(l.y, h.y, bounds + (kGridSlabs + 1));
        const int tz = slab_tri(l.z, h.z, bounds + 2 * (kGridSlabs + 1));
        edge_tri[(size_t)warp * G + g] = (tx < 0 || ty < 0 || tz < 0) ? -1 : (tx | (ty << 10) | (tz << 20));
    }
}

// ------------------------------------------------------------------ 6. check
// Whole warp: does link group g's bounding sphere at sample k hit any of the
// environment's np primitives (the reference's gate, every primitive)?
template <class M>
__device__ __forceinline__ bool bound_hits_any(const float4* __restrict__ table, size_t row0, int k, int g,
                                               const float4* prim, int np) {
    const int lane = threadIdx.x & 31;
    float4 b = table[table_index<M>(row0 + (size_t)k, g)];
    b.w += kEnvInflate;
    bool any = false;
    for (int p = lane; p < np; p += 32) any |= sphere_hits_prim(b, prim + p * kPrimF4);
    return __any_sync(kFull, any);
}

// Learned order, rank r -> sample index: segments in the order perm gives
// (descending MLP score), each walked from its last sample back to its first.
// The MLP scores a segment at its last sample (queue_features_kernel), so the
// scored sample is the first one checked; a collision that starts inside an
// edge whose start is free usually extends to the edge's end, so within a
// segment the later samples are the likelier hits.
__device__ __forceinline__ int learned_rank_to_sample(const uint8_t* perm, int r) {
    return (int)perm[r >> 3] * kSegment + (kSegment - 1 - (r & (kSegment - 1)));
}

// Inline learned order: a permutation pi of the 32 lane blocks (block t =
// samples t n .. t n + n - 1, the samples the reference's lane t checks) with
// pi[0] = 0; rank r -> sample pi[r % 32] n + r / 32, so every round visits the
// blocks in learned order, round 0 first (the reference's coarse sweep,
// re-prioritised), starting with sample 0 (where most colliding pairs collide).
// Each lane holds pi[lane]; the walk fetches pi[r % 32] by shuffle.

// Per-pair walk counts (32 bits: a pair walks at most 32 n C items, far below
// 2^32; the registers and adds are paid on every walk, counting or not).
struct WalkStats {
    unsigned chunks = 0, gates = 0, leaf = 0;
};

// Leaf steps of the overhang-aware walk fetch their item's fields (pair code,
// gate bit, leaf offset) with one shuffle where that measured faster: Fetch
// (+1.5 %); Baxter's larger walk spills more with the packed value live (-1.5 %)
// and keeps one shuffle per field.  The group count separates the two models.
template <class M>
constexpr bool pack_overhang_leaf() {
    return M::num_env_groups <= 16;
}

// Lane g's copy of link group g's leaf range, packed (first leaf | leaf count
// << 16).  The walk fetches a group's range with one shuffle: its lanes hold
// items of different groups, and indexing __constant__ memory with a
// lane-dependent group serialises the access once per distinct group.
struct GroupLanes {
    int fc;
    float cert;  // lane g: group g's certain-hit radius
};

template <class M>
__device__ __forceinline__ GroupLanes group_lanes() {
    const DevTables<M>& T = tab<M>();
    const int g = min(threadIdx.x & 31, M::num_env_groups - 1);
    const int first = T.leaf_begin[g];
    GroupLanes r;
    r.fc = first | ((T.leaf_begin[g + 1] - first) << 16);
    r.cert = T.cert_r[g];
    return r;
}

// Whole warp: walk (sample rank, pair) items 32 at a time in check order --
// plain reference order, or with `perm` the edge's segments in learned order --
// and return whether some item collides.  Items [w_begin, w_end) are walked
// (w_end < 0: all).  MODE 1 (probe) with overhang: after the chunk that
// completes rank 0, when at least queue_min_items remain, the whole warp calls
// queue(); if that queues the pair, the walk stops with `undecided` set,
// otherwise it goes on in plain order (robots without overhang make that
// decision in check_pair, between two walks).
// Each chunk tests the bounds (one per item); the leaf work of the items whose
// bound hit is then flattened over the warp (item j owns leaf slots
// [incl_j - cnt_j, incl_j)) and the warp stops at the first step with a hit.
// MODE 2 (finish): the CTA's warps split the pair -- this warp walks the
// chunks at w_begin, w_begin + 32 stride, ... and all stop once one of them
// sets *stop.
template <class M, int MODE, class Queue>
__device__ __forceinline__ bool walk_pairs(const float4* __restrict__ table, size_t row0, int n, int C,
                                           const uint16_t* pairs, const float4* prim, int np, const uint8_t* perm,
                                           int queue_min_items, const GroupLanes& GL, bool& undecided,
                                           WalkStats& st, Queue&& queue, int w_begin = 0, int w_end = -1,
                                           int stride = 1, volatile int* stop = nullptr) {
    constexpr int G = M::num_env_groups;
    constexpr int GB = group_bits<M>();
    constexpr bool kOver = has_overhang<M>();
    // rank -> sample: reference order (MODE 0, 1, or no perm), learned order
    // (MODE 2, 3), inline learned order (MODE 4: perm = the pair's 32-block
    // permutation, block fetched by a shuffle every lane executes).
    const int pi = MODE == 4 && perm ? (int)perm[threadIdx.x & 31] : (int)(threadIdx.x & 31);
    auto block_of = [&](int rr) {
        if constexpr (MODE == 4) return __shfl_sync(kFull, pi, rr & (kLanes - 1));
        return rr & (kLanes - 1);
    };
    auto sample_of = [&](int rr, int blk) {
        if constexpr (MODE == 0 || MODE == 1 || MODE == 4) {
            return blk * n + (rr >> 5);
        } else {
            return perm ? learned_rank_to_sample(perm, rr) : reference_rank_to_sample(rr, n);
        }
    };
    const int lane = threadIdx.x & 31;
    const int total = kLanes * n * C;
    const int w_last = w_end < 0 ? total : w_end;
    const int w_step = 32 * stride;
    int dr, dc, r, c;
    if (MODE != 2 && w_begin == 0) {
        // a / C for a <= 32 and 1 <= C <= kPairCap: floor((a + 0.5) / C) in FP32 is
        // exact (the quotient stays >= 1 / 2048 away from an integer), and cheaper
        // than an integer division by a runtime divisor.
        const float inv_c = __frcp_rn((float)C);
        dr = (int)(32.5f * inv_c);
        dc = 32 - dr * C;
        r = (int)(((float)lane + 0.5f) * inv_c);
        c = lane - r * C;
    } else {
        dr = w_step / C;
        dc = w_step - dr * C;
        r = (w_begin + lane) / C;
        c = w_begin + lane - r * C;
    }
    bool collide = false;
    {
        for (int w0 = w_begin; w0 < w_last; w0 += w_step) {
            if constexpr (MODE == 2) {  // another warp of the CTA found a hit
                int s = 0;
                if (lane == 0) s = *stop;
                if (__shfl_sync(kFull, s, 0)) break;
            }
            bool gate = false, cert = false;
            int g = 0, p = 0, k = 0, cnt = 0, first = 0;
            if constexpr (!kOver) {
                // c < C on every lane, also past the last item: the pair is decoded and
                // its group's leaf range fetched by shuffle on every lane (measured
                // faster for Panda than lane-indexed constant memory), the table and
                // the primitive read only for live items.
                const uint32_t pr = pairs[c];
                g = (int)(pr & ((1u << GB) - 1u));
                p = (int)(pr >> GB);
                const int fc = __shfl_sync(kFull, GL.fc, g);
                const float cr = __shfl_sync(kFull, GL.cert, g);
                first = fc & 0xffff;
                const int gcnt = fc >> 16;
                const int blk = block_of(r);
                if (w0 + lane < total) {
                    k = sample_of(r, blk);
                    float4 bs = table[table_index<M>(row0 + (size_t)k, g)];
                    bs.w += kEnvInflate;
                    float rho;
                    const float d2 = prim_core_d2(bs, prim + p * kPrimF4, &rho);
                    const float rr = bs.w + rho;
                    gate = d2 - rr * rr < 0.0f;
                    // the bound's centre close enough to the core proves a leaf hit
                    const float rc = rho + cr;
                    cert = cr > 0.0f && d2 - rc * rc < 0.0f;
                    cnt = gate ? gcnt : 0;
                }
            } else {
                // The overhang-aware walk reads its group fields from constant memory,
                // which leaves its longer body the registers it needs (measured faster
                // for Fetch and Baxter).
                const DevTables<M>& T = tab<M>();
                const int blk = block_of(r);
                if (w0 + lane < total) {
                    k = sample_of(r, blk);
                    const uint32_t pr = pairs[c];
                    g = (int)(pr & ((1u << GB) - 1u));
                    p = (int)(pr >> GB);
                    float4 bs = table[table_index<M>(row0 + (size_t)k, g)];
                    bs.w += kEnvInflate;
                    float rho;
                    const float d2 = prim_core_d2(bs, prim + p * kPrimF4, &rho);
                    const float rr = bs.w + rho;
                    gate = d2 - rr * rr < 0.0f;
                    const float rc = rho + T.cert_r[g];
                    cert = T.cert_r[g] > 0.0f && d2 - rc * rc < 0.0f;
                    cnt = gate ? T.leaf_begin[g + 1] - T.leaf_begin[g] : 0;
                    // overhanging leaves (listed first) near a primitive the bound misses
                    if (!gate && T.over_count[g] > 0) {
                        const float rp = rr + T.cull_pad[g];
                        if (d2 - rp * rp < 0.0f) cnt = T.over_count[g];
                    }
                }
                first = T.leaf_begin[g];
            }
            ++st.chunks;
            if (__any_sync(kFull, cert)) {  // a leaf hit is certain: no leaf step
                collide = true;
                break;
            }
            if (__any_sync(kFull, cnt > 0)) {
                ++st.gates;
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(kFull, incl, o);
                    if (lane >= o) incl += y;
                }
                const int L = __shfl_sync(kFull, incl, 31);
                // Without overhang a slot needs only its item's sample, primitive
                // and leaf offset: p | (first - exclusive count) << 12, one shuffle.
                int dp = 0;
                if constexpr (!kOver) {
                    static_assert(max_prims_of<M>() < 4096, "primitive index packs into 12 bits");
                    dp = (int)(((unsigned)(first - (incl - cnt)) << 12) | (unsigned)p);
                } else if constexpr (pack_overhang_leaf<M>()) {
                    // the 16-bit pair code (p << GB | g), the gate bit, the leaf offset
                    dp = (int)(((unsigned)(first - (incl - cnt)) << 17) | ((unsigned)gate << 16) |
                               ((unsigned)p << GB) | (unsigned)g);
                }
                for (int t0 = 0; t0 < L; t0 += 32) {
                    const int t = t0 + lane;
                    // owner j: the first lane whose inclusive count exceeds t
                    int j = 0;
#pragma unroll
                    for (int step = 16; step; step >>= 1) {
                        const int v = __shfl_sync(kFull, incl, j + step - 1);
                        if (v <= t) j += step;
                    }
                    int j_k, j_p, leaf, jd = 0;
                    if constexpr (!kOver) {
                        jd = __shfl_sync(kFull, dp, j);
                        j_k = __shfl_sync(kFull, k, j);
                        j_p = jd & 4095;
                        leaf = t + (jd >> 12);
                    } else if constexpr (pack_overhang_leaf<M>()) {
                        jd = __shfl_sync(kFull, dp, j);
                        j_k = __shfl_sync(kFull, k, j);
                        j_p = (jd & 0xffff) >> GB;
                        leaf = t + (jd >> 17);
                    } else {
                        const int j_incl = __shfl_sync(kFull, incl, j);
                        const int j_cnt = __shfl_sync(kFull, cnt, j);
                        const int j_first = __shfl_sync(kFull, first, j);
                        j_k = __shfl_sync(kFull, k, j);
                        j_p = __shfl_sync(kFull, p, j);
                        leaf = j_first + (t - (j_incl - j_cnt));
                    }
                    bool hit = false;
                    if (t < L) {
                        float4 ls = table[table_index<M>(row0 + (size_t)j_k, G + leaf)];
                        ls.w += kEnvInflate;
                        hit = sphere_hits_prim(ls, prim + j_p * kPrimF4);
                    }
                    ++st.leaf;
                    if constexpr (kOver) {
                        const bool j_gate = pack_overhang_leaf<M>() ? ((jd >> 16) & 1) != 0
                                                                    : __shfl_sync(kFull, (int)gate, j) != 0;
                        if (__any_sync(kFull, hit && j_gate)) {
                            collide = true;
                            break;
                        }
                        // Hits of overhanging leaves whose bound missed this primitive:
                        // they count once the bound hits some primitive at that sample.
                        const int j_g = pack_overhang_leaf<M>() ? (jd & ((1 << GB) - 1)) : __shfl_sync(kFull, g, j);
                        uint32_t pend = __ballot_sync(kFull, hit);
                        while (pend) {
                            const int u = __ffs(pend) - 1;
                            const int uk = __shfl_sync(kFull, j_k, u);
                            const int ug = __shfl_sync(kFull, j_g, u);
                            if (bound_hits_any<M>(table, row0, uk, ug, prim, np)) {
                                collide = true;
                                break;
                            }
                            pend &= ~__ballot_sync(kFull, j_k == uk && j_g == ug);
                        }
                        if (collide) break;
                    } else {
                        if (__any_sync(kFull, hit)) {
                            collide = true;
                            break;
                        }
                    }
                }
                if (collide) break;
            }
            // Probe (overhang-aware walk): the queue decision stays inside the
            // loop, measured 5 % faster for Baxter than a separate first walk.
            if constexpr (MODE == 1 && kOver) {
                if (w0 == (((C - 1) >> 5) << 5) && total - (w0 + 32) >= queue_min_items && queue()) {
                    undecided = true;
                    break;
                }
            }
            c += dc;
            r += dr;
            if (c >= C) {
                c -= C;
                ++r;
            }
        }
    }
    if constexpr (MODE == 2) {
        if (collide && lane == 0) *stop = 1;
    }
    return collide;
}

// Learned order, whole warp: perm_buf[rank] = segment, the edge's nseg <= 64
// segments in descending MLP score (scores[0 .. nseg)), ties by index, NaN
// last; returns segment 0's rank.
__device__ __forceinline__ int rank_segments(const float* scores, int nseg, uint8_t* perm_buf) {
    const int lane = threadIdx.x & 31;
    float v0 = lane < nseg ? scores[lane] : -INFINITY;
    float v1 = lane + 32 < nseg ? scores[lane + 32] : -INFINITY;
    v0 = isnan(v0) ? -INFINITY : v0;
    v1 = isnan(v1) ? -INFINITY : v1;
    int rank0 = 0, rank1 = 0;
    for (int i = 0; i < nseg; ++i) {
        const float vi = __shfl_sync(kFull, i < 32 ? v0 : v1, i & 31);
        rank0 += (vi > v0 || (vi == v0 && i < lane)) ? 1 : 0;
        rank1 += (vi > v1 || (vi == v1 && i < lane + 32)) ? 1 : 0;
    }
    if (lane < nseg) perm_buf[rank0] = (uint8_t)lane;
    if (lane + 32 < nseg) perm_buf[rank1] = (uint8_t)(lane + 32);
    return __shfl_sync(kFull, rank0, 0);
}

__device__ __forceinline__ void learned_perm(const CheckParams& P, int seg_row, int nseg, uint8_t* perm_buf) {
    rank_segments(P.logits + seg_row, nseg, perm_buf);
}

// Learned-order queue: lane 0 of a probing warp reserves a queue entry and the
// 4 n MLP rows of the pair's segments with one 64-bit atomic on q_head (entries
// in the high word, rows in the low word).  Returns the pair's first MLP row,
// or -1 when the pair keeps the plain order (more than kMaxSegments segments,
// or the row budget or the queue spent) and the probe walks on.  The low word
// only grows while it is at most row_cap, so it stays far below 2^32.
__device__ __forceinline__ int queue_pair(const CheckParams& P, int e, int env, int n) {
    const int rows = 4 * n;
    if (rows > kMaxSegments) return -1;
    const unsigned used = *reinterpret_cast<volatile const unsigned*>(P.q_head);
    if ((long long)used + rows > P.row_cap) return -1;
    const unsigned long long old = atomicAdd(P.q_head, (1ull << 32) | (unsigned long long)rows);
    const long long idx = (long long)(old >> 32);
    if (idx >= P.q_cap) return -1;
    const unsigned ro = (unsigned)old;
    const int r = (long long)ro + rows <= P.row_cap ? (int)ro : -1;
    P.q_pairs[idx] = make_int2(e, env);
    P.q_rows[idx] = r;
    return r;
}

// Inline learned order of pair (env, e): the 32-block permutation scored for
// the environment's cluster.
__device__ __forceinline__ const uint8_t* inline_perm(const CheckParams& P, int env, int e) {
    return P.perms + ((size_t)P.env_cluster[env] * P.num_edges + e) * kLanes;
}

// One (environment, edge) pair, whole warp: cull, pair-list compaction and the
// walk.  MODE 0: plain order, full walk.  MODE 1 (learned pipeline, phase 1):
// plain order; a pair still undecided once rank 0 (its first sample) is walked may be
// queued (with MLP rows for its segments) instead of getting a verdict.  MODE 2
// (phase 3): a queued pair (first MLP row seg_row) walked in descending
// segment score, its chunks split over the CTA's warps; MODE 3 (phase 3, one
// warp per pair): the same walk by this warp alone, which writes the verdict.
// `prim` holds the environment's records (shared or global memory), `masks`
// its cull masks, W 64-bit words per mask.
template <class M, int MODE>
__device__ __forceinline__ void check_pair(const CheckParams& P, int env, int e, int seg_row, const float4* prim,
                                           const uint64_t* __restrict__ masks, int np, int W, uint16_t* pairs,
                                           uint8_t* perm_buf, const GroupLanes& GL, int chunk0 = 0, int stride = 1,
                                           volatile int* stop = nullptr) {
    constexpr int G = M::num_env_groups;
    constexpr int GB = group_bits<M>();
    const int lane = threadIdx.x & 31;
    const int K = P.pairs_per_warp;
    uint8_t* out = P.results + (size_t)e * P.num_envs + env;
    const int self = P.edge_self[e];
    if (np == 0 || self) {  // a self-colliding sample collides in every environment
        if (lane == 0) {
            *out = self ? 1 : 0;
            if (MODE == 2 && self) *stop = 1;  // the finish kernel writes s_hit as the verdict
        }
        return;
    }
    // Cull: lane g < G takes link g's slab ranges on the set's grid (computed
    // once per edge) and ANDs the environment's three masks over them.
    const int code = lane < G ? P.edge_tri[(size_t)e * G + lane] : -1;
    // Word w of link g's candidate mask (only the packed code stays live
    // across the walk; the three offsets are re-derived where needed).
    auto mask_word = [&](int w) {
        const int tx = code & 1023, ty = (code >> 10) & 1023, tz = code >> 20;
        return __ldg(masks + tx * W + w) & __ldg(masks + (kGridTri + ty) * W + w) &
               __ldg(masks + (2 * kGridTri + tz) * W + w);
    };
    // Compact the surviving (primitive, link) pairs, link-major: lane g counts
    // link g's candidates, an exclusive warp scan gives each link its offset,
    // and every lane writes its own link's pairs in primitive order.
    int cnt = 0;
    if (code >= 0)
        for (int w = 0; w < W; ++w) cnt += __popcll(mask_word(w));
    int off = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, off, o);
        if (lane >= o) off += y;
    }
    const int C = __shfl_sync(kFull, off, 31);
    off -= cnt;

    bool collide = false, undecided = false;
    WalkStats st;
    // Pair list entries [seg0, seg1): lane g writes link g's candidates that
    // fall in the range.
    auto write_seg = [&](int seg0, int seg1) {
        if (cnt > 0 && off < seg1 && off + cnt > seg0) {
            int idx = off;
            for (int w = 0; w < W && idx < seg1; ++w) {
                uint64_t m = mask_word(w);
                while (m && idx < seg1) {
                    const int b = __ffsll((long long)m) - 1;
                    if (idx >= seg0) pairs[idx - seg0] = (uint16_t)(((w * 64 + b) << GB) | lane);
                    ++idx;
                    m &= m - 1;
                }
            }
        }
        __syncwarp();
    };
    auto queue = [&]() {
        int ro = -1;
        if (lane == 0) ro = queue_pair(P, e, env, P.steps[e]);
        return __shfl_sync(kFull, ro, 0) >= 0;
    };
    auto walk_seg = [&](int Cs) {
        const int n = P.steps[e];
        const size_t row0 = (size_t)P.offs[e];
        // Learned order: rank the edge's 4 n segments by their MLP score
        // (descending, ties by index; NaN scores last).
        const int nseg = 4 * n;
        const bool learned = (MODE == 2 || MODE == 3) && seg_row >= 0 && nseg <= kMaxSegments;
        if (learned) {
            learned_perm(P, seg_row, nseg, perm_buf);
            __syncwarp();
        }
        if constexpr (MODE == 1 && !has_overhang<M>()) {
            // Probe: walk up to the chunk that completes rank 0 (the edge's first
            // sample against every candidate, where most colliding pairs
            // collide); when at least queue_min_items items remain, queue the
            // pair for the learned order or, if queue() declines, walk on.  Two
            // plain walks, so no chunk of either pays for the decision.
            const int total = kLanes * n * Cs;
            const int w_dec = (((Cs - 1) >> 5) << 5) + 32;
            if (total - w_dec >= P.queue_min_items) {
                collide = walk_pairs<M, 0>(P.table, row0, n, Cs, pairs, prim, np, nullptr, 0, GL, undecided, st,
                                           queue, 0, w_dec);
                if (!collide) {
                    if (queue())
                        undecided = true;
                    else
                        collide = walk_pairs<M, 0>(P.table, row0, n, Cs, pairs, prim, np, nullptr, 0, GL, undecided,
                                                   st, queue, w_dec);
                }
            } else {
                collide = walk_pairs<M, 0>(P.table, row0, n, Cs, pairs, prim, np, nullptr, 0, GL, undecided, st,
                                           queue);
            }
        } else if constexpr (MODE == 4) {
            collide = walk_pairs<M, 4>(P.table, row0, n, Cs, pairs, prim, np, inline_perm(P, env, e), 0, GL,
                                       undecided, st, queue);
        } else {
            collide = walk_pairs<M, MODE>(P.table, row0, n, Cs, pairs, prim, np, learned ? perm_buf : nullptr,
                                          P.queue_min_items, GL, undecided, st, queue, 32 * chunk0, -1, stride,
                                          stop);
        }
        __syncwarp();  // every lane is done with this segment's pairs
    };
    // Robots whose leaves all lie inside their bounds have a small walk: a
    // separate copy for the usual single-segment case keeps the segment
    // bookkeeping out of it.  The overhang-aware walk stays in one copy.
    bool single = false;
    if constexpr (!has_overhang<M>()) single = C > 0 && C <= K;
    // The whole list fits the buffer (the usual case): no segment bounds to test
    // while writing.
    auto write_all = [&]() {
        if (cnt > 0) {
            int idx = off;
            for (int w = 0; w < W; ++w) {
                uint64_t m = mask_word(w);
                while (m) {
                    const int b = __ffsll((long long)m) - 1;
                    pairs[idx++] = (uint16_t)(((w * 64 + b) << GB) | lane);
                    m &= m - 1;
                }
            }
        }
        __syncwarp();
    };
    if (single) {
        write_all();
        walk_seg(C);
    } else {
        for (int seg0 = 0; seg0 < C && !collide && !undecided; seg0 += K) {
            const int seg1 = min(C, seg0 + K);
            if (C <= K)
                write_all();
            else
                write_seg(seg0, seg1);
            walk_seg(seg1 - seg0);
        }
    }
    if (MODE == 1 && undecided) return;  // queued: the finish pass writes the verdict
    if (MODE == 2) {  // the CTA's warps split the pair: the finish kernel writes the verdict
        if (lane == 0 && P.counters) {
            if (chunk0 == 0) atomicAdd(P.counters + 1, (unsigned long long)C);
            atomicAdd(P.counters + 2, (unsigned long long)st.chunks);
            atomicAdd(P.counters + 3, (unsigned long long)st.gates);
            atomicAdd(P.counters + 4, (unsigned long long)st.leaf);
        }
        return;
    }
    if (lane == 0) {
        *out = collide ? 1 : 0;
        if (P.counters) {
            atomicAdd(P.counters + 0, 1ull);
            atomicAdd(P.counters + 1, (unsigned long long)C);
            atomicAdd(P.counters + 2, (unsigned long long)st.chunks);
            atomicAdd(P.counters + 3, (unsigned long long)st.gates);
            atomicAdd(P.counters + 4, (unsigned long long)st.leaf);
            atomicAdd(P.counters + 5, collide ? 1ull : 0ull);
        }
    }
}

// Pairs whose cull and compaction one warp does together: lanes are grouped G
// to a pair (Panda 10 -> 3 pairs, Fetch 15 -> 2, Baxter 32 -> 1), so the
// per-pair set-up -- slab-range loads, mask ANDs, counts, the scan and the
// list writes -- runs on 30 (or 30, 32) lanes instead of G.
template <class M>
constexpr int pairs_per_setup() {
    return kLanes / M::num_env_groups;
}

// The walk of one pair whose whole candidate list is in `pairs` (C entries,
// C <= pairs_per_warp), whole warp, and its verdict: MODE 0 plain order;
// MODE 1 probe (plain walk of rank 0, then queue the pair or walk on); MODE 4
// inline learned order.
template <class M, int MODE>
__device__ __forceinline__ void walk_listed_pair(const CheckParams& P, int env, int e, int C, const uint16_t* pairs,
                                                 const float4* prim, int np, const GroupLanes& GL) {
    const int lane = threadIdx.x & 31;
    const int n = P.steps[e];
    const size_t row0 = (size_t)P.offs[e];
    bool collide = false, undecided = false;
    WalkStats st;
    auto queue = [&]() {
        int ro = -1;
        if (lane == 0) ro = queue_pair(P, e, env, n);
        return __shfl_sync(kFull, ro, 0) >= 0;
    };
    if constexpr (MODE == 1 && !has_overhang<M>()) {
        // Probe, as in check_pair: two plain walks split at the chunk that
        // completes rank 0, the queue decision between them.
        const int total = kLanes * n * C;
        const int w_dec = (((C - 1) >> 5) << 5) + 32;
        if (total - w_dec >= P.queue_min_items) {
            collide = walk_pairs<M, 0>(P.table, row0, n, C, pairs, prim, np, nullptr, 0, GL, undecided, st, queue, 0,
                                       w_dec);
            if (!collide) {
                if (queue())
                    undecided = true;
                else
                    collide = walk_pairs<M, 0>(P.table, row0, n, C, pairs, prim, np, nullptr, 0, GL, undecided, st,
                                               queue, w_dec);
            }
        } else {
            collide = walk_pairs<M, 0>(P.table, row0, n, C, pairs, prim, np, nullptr, 0, GL, undecided, st, queue);
        }
    } else if constexpr (MODE == 4) {
        collide = walk_pairs<M, 4>(P.table, row0, n, C, pairs, prim, np, inline_perm(P, env, e), 0, GL, undecided,
                                   st, queue);
    } else {
        collide = walk_pairs<M, MODE>(P.table, row0, n, C, pairs, prim, np, nullptr, P.queue_min_items, GL, undecided,
                                      st, queue);
    }
    if (MODE == 1 && undecided) return;  // queued: the finish pass walks, counts and writes the verdict
    if (lane == 0) {
        P.results[(size_t)e * P.num_envs + env] = collide ? 1 : 0;
        if (P.counters) {
            atomicAdd(P.counters + 0, 1ull);
            atomicAdd(P.counters + 1, (unsigned long long)C);
            atomicAdd(P.counters + 2, (unsigned long long)st.chunks);
            atomicAdd(P.counters + 3, (unsigned long long)st.gates);
            atomicAdd(P.counters + 4, (unsigned long long)st.leaf);
            atomicAdd(P.counters + 5, collide ? 1ull : 0ull);
        }
    }
}

// Plain order with 16 lanes per walking pair (MODE 5; robots whose leaves lie
// inside their bounds): the warp's two halves walk two listed pairs at once,
// 16 (sample rank, candidate) items a step each, in the reference's order.
// The leaf work of a step is flattened inside each half; a half whose pair is
// decided (a hit, or every item walked) writes the verdict and takes the next
// pair of the walk list wt[0 .. nwalk).  A pair that collides in its first 16
// items -- most of them -- then costs half a warp step instead of a whole one.
template <class M, int SUB>
__device__ __forceinline__ void walk_halves(const CheckParams& P, int env, int e0, int nwalk, const int (&wt)[SUB],
                                            const int (&Cs)[SUB], const int (&base)[SUB], const uint16_t* pairs,
                                            const float4* prim, const GroupLanes& GL) {
    static_assert(!has_overhang<M>(), "the half-warp walk covers robots whose leaves lie inside their bounds");
    constexpr int G = M::num_env_groups;
    constexpr int GB = group_bits<M>();
    constexpr int H = 16;
    const int lane = threadIdx.x & 31, h = lane >> 4, hl = lane & (H - 1);
    const unsigned hmask = h ? 0xffff0000u : 0x0000ffffu;
    int t = -1, C = 1, bse = 0, n = 1, total = 0, w0 = 0, r = 0, c = 0, dr = 0, dc = 0, e = e0, row0 = 0;
    WalkStats st;
    auto take = [&](int idx) {
        int tt = -1;
#pragma unroll
        for (int u = 0; u < SUB; ++u)
            if (u == idx && u < nwalk) tt = wt[u];
        t = tt;
        if (t >= 0) {
            int cc = 1, bb = 0;
#pragma unroll
            for (int u = 0; u < SUB; ++u)
                if (u == t) {
                    cc = Cs[u];
                    bb = base[u];
                }
            C = cc;
            bse = bb;
            e = e0 + t;
            n = P.steps[e];
            row0 = P.offs[e];
            total = kLanes * n * C;
            w0 = 0;
            // a / C for a <= 16 in FP32, exact as in walk_pairs
            const float inv_c = __frcp_rn((float)C);
            dr = (int)(16.5f * inv_c);
            dc = H - dr * C;
            r = (int)(((float)hl + 0.5f) * inv_c);
            c = hl - r * C;
            st = WalkStats();
        }
    };
    take(h);
    int nxt = 2;
    // Bound on the loop (the warp-uniform step count): every step walks 16
    // items of each live pair or ends one, so a group of pairs needs far fewer;
    // past it the warp flags the error and leaves.
    unsigned steps_left = 1u << 24;
    for (;;) {
        const bool act = t >= 0;
        if (!__any_sync(kFull, act)) break;
        if (--steps_left == 0) {
            if (lane == 0) atomicOr(P.error_flag, 4);
            break;
        }
        const uint32_t pr = act ? (uint32_t)pairs[bse + c] : 0u;
        const int g = (int)(pr & ((1u << GB) - 1u));
        const int p = (int)(pr >> GB);
        const int fc = __shfl_sync(kFull, GL.fc, g);
        const int first = fc & 0xffff, gcnt = fc >> 16;
        int k = 0, cnt = 0;
        if (act && w0 + hl < total) {
            k = reference_rank_to_sample(r, n);
            float4 bs = P.table[table_index<M>((size_t)(row0 + k), g)];
            bs.w += kEnvInflate;
            cnt = sphere_hits_prim(bs, prim + p * kPrimF4) ? gcnt : 0;
        }
        if (act) ++st.chunks;
        bool hitp = false;
        const unsigned gates = __ballot_sync(kFull, cnt > 0);
        if (gates) {
            if (gates & hmask) ++st.gates;
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < H; o <<= 1) {
                const int y = __shfl_up_sync(kFull, incl, o, H);
                if (hl >= o) incl += y;
            }
            const int L = __shfl_sync(kFull, incl, H - 1, H);
            const int Lw = max(L, __shfl_xor_sync(kFull, L, 16));
            // a slot's item: its sample, primitive and leaf offset (first - exclusive count)
            static_assert(max_prims_of<M>() < 4096, "primitive index packs into 12 bits");
            const int dp = (int)(((unsigned)(first - (incl - cnt)) << 12) | (unsigned)p);
            for (int t0 = 0; t0 < Lw; t0 += H) {
                const int tt = t0 + hl;
                int j = 0;  // owner: the first lane of the half whose inclusive count exceeds tt
#pragma unroll
                for (int step = H / 2; step; step >>= 1) {
                    const int v = __shfl_sync(kFull, incl, j + step - 1, H);
                    if (v <= tt) j += step;
                }
                const int jd = __shfl_sync(kFull, dp, j, H);
                const int jk = __shfl_sync(kFull, k, j, H);
                bool hit = false;
                if (tt < L) {
                    float4 ls = P.table[table_index<M>((size_t)(row0 + jk), G + tt + (jd >> 12))];
                    ls.w += kEnvInflate;
                    hit = sphere_hits_prim(ls, prim + (jd & 4095) * kPrimF4);
                }
                if (t0 < L) ++st.leaf;
                // the ballot on its own statement: every lane must reach it, so it
                // must not sit behind a short-circuiting ||
                const unsigned hb = __ballot_sync(kFull, hit);
                hitp = hitp || (hb & hmask) != 0;
                if (__all_sync(kFull, hitp || t0 + H >= L)) break;  // every half hit or out of slots
            }
        }
        bool fin = false;
        if (act) {
            if (hitp) {
                fin = true;
            } else {
                w0 += H;
                c += dc;
                r += dr;
                if (c >= C) {
                    c -= C;
                    ++r;
                }
                fin = w0 >= total;
            }
        }
        if (fin && hl == 0) {
            P.results[(size_t)e * P.num_envs + env] = hitp ? 1 : 0;
            if (P.counters) {
                atomicAdd(P.counters + 0, 1ull);
                atomicAdd(P.counters + 1, (unsigned long long)C);
                atomicAdd(P.counters + 2, (unsigned long long)st.chunks);
                atomicAdd(P.counters + 3, (unsigned long long)st.gates);
                atomicAdd(P.counters + 4, (unsigned long long)st.leaf);
                atomicAdd(P.counters + 5, hitp ? 1ull : 0ull);
            }
        }
        // next pairs, in half order, the same on every lane
        const unsigned fb = __ballot_sync(kFull, fin && hl == 0);
        const int f0 = (int)(fb & 1u), f1 = (int)((fb >> 16) & 1u);
        const int i0 = nxt, i1 = nxt + f0;
        nxt += f0 + f1;
        if (fin) take(h ? i1 : i0);
    }
}

// Pairs (env, e0 .. e0 + count - 1), count <= pairs_per_setup<M>(), whole
// warp: lane group s = lane / G culls pair s (lane g of the group ANDs link
// g's three masks), a scan inside each group gives every link its offset,
// the groups' lists are laid out one after another in `pairs` and written in
// one pass; then the warp walks the pairs one at a time.  When the lists do
// not fit the warp's buffer together, each pair goes through check_pair
// (segments).
template <class M, int MODE>
__device__ __forceinline__ void check_pair_group(const CheckParams& P, int env, int e0, int count, const float4* prim,
                                                 const uint64_t* __restrict__ masks, int np, int W, uint16_t* pairs,
                                                 const GroupLanes& GL) {
    constexpr int G = M::num_env_groups;
    constexpr int GB = group_bits<M>();
    constexpr int SUB = pairs_per_setup<M>();
    const int lane = threadIdx.x & 31;
    const int sub = lane / G;
    const int g = lane - sub * G;
    const bool live = sub < count;
    const int e = e0 + (live ? sub : 0);
    const int self = live ? P.edge_self[e] : 1;
    const int code = (live && !self && np > 0) ? P.edge_tri[(size_t)e * G + g] : -1;
    auto mask_word = [&](int w) {
        const int tx = code & 1023, ty = (code >> 10) & 1023, tz = code >> 20;
        return __ldg(masks + tx * W + w) & __ldg(masks + (kGridTri + ty) * W + w) &
               __ldg(masks + (2 * kGridTri + tz) * W + w);
    };
    // One mask word (np <= 64, the common case) stays in registers for the
    // list writes; more words are re-read there.
    int cnt = 0;
    uint64_t m1 = 0;
    if (code >= 0) {
        if (W == 1) {
            m1 = mask_word(0);
            cnt = __popcll(m1);
        } else {
            for (int w = 0; w < W; ++w) cnt += __popcll(mask_word(w));
        }
    }
    // inclusive scan inside each group of G lanes
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
        const int y = __shfl_up_sync(kFull, inc, o);
        if (g >= o) inc += y;
    }
    // every pair's candidate count and list base
    int Cs[SUB], base[SUB], total = 0;
#pragma unroll
    for (int t = 0; t < SUB; ++t) {
        Cs[t] = __shfl_sync(kFull, inc, t * G + G - 1);
        base[t] = total;
        total += t < count ? Cs[t] : 0;
    }
    constexpr int PAIR_MODE = MODE == 5 ? 0 : MODE;
    if (total > P.pairs_per_warp) {
        for (int t = 0; t < count; ++t)
            check_pair<M, PAIR_MODE>(P, env, e0 + t, -1, prim, masks, np, W, pairs, nullptr, GL);
        return;
    }
    if (cnt > 0) {
        int idx = inc - cnt;
#pragma unroll
        for (int t = 0; t < SUB; ++t)
            if (t == sub) idx += base[t];
        if (W == 1) {  // 32-bit halves: cheaper bit steps than 64-bit ones
            uint32_t lo = (uint32_t)m1, hi = (uint32_t)(m1 >> 32);
            while (lo) {
                pairs[idx++] = (uint16_t)(((__ffs((int)lo) - 1) << GB) | g);
                lo &= lo - 1u;
            }
            while (hi) {
                pairs[idx++] = (uint16_t)(((__ffs((int)hi) + 31) << GB) | g);
                hi &= hi - 1u;
            }
        } else {
            for (int w = 0; w < W; ++w) {
                uint64_t m = mask_word(w);
                while (m) {
                    const int b = __ffsll((long long)m) - 1;
                    pairs[idx++] = (uint16_t)(((w * 64 + b) << GB) | g);
                    m &= m - 1;
                }
            }
        }
    }
    __syncwarp();
    if constexpr (MODE == 5) {
        // the pairs decided without a walk first, the rest walked by half-warps
        int wt[SUB];
        int nwalk = 0;
#pragma unroll
        for (int t = 0; t < SUB; ++t) wt[t] = -1;
#pragma unroll
        for (int t = 0; t < SUB; ++t) {
            if (t >= count) continue;  // warp-uniform
            const int et = e0 + t;
            const int self_t = __shfl_sync(kFull, self, t * G);
            if (np == 0 || self_t) {
                if (lane == 0) P.results[(size_t)et * P.num_envs + env] = self_t ? 1 : 0;
                continue;
            }
            if (Cs[t] == 0) {
                if (lane == 0) {
                    P.results[(size_t)et * P.num_envs + env] = 0;
                    if (P.counters) atomicAdd(P.counters + 0, 1ull);
                }
                continue;
            }
#pragma unroll
            for (int u = 0; u < SUB; ++u)
                if (u == nwalk) wt[u] = t;
            ++nwalk;
        }
        walk_halves<M, SUB>(P, env, e0, nwalk, wt, Cs, base, pairs, prim, GL);
    } else {
#pragma unroll 1
    for (int t = 0; t < count; ++t) {
        const int et = e0 + t;
        const int self_t = __shfl_sync(kFull, self, t * G);
        if (np == 0 || self_t) {  // decided without a walk (not counted as walked, as in check_pair)
            if (lane == 0) P.results[(size_t)et * P.num_envs + env] = self_t ? 1 : 0;
            continue;
        }
        if (Cs[t] == 0) {  // nothing survives the cull: free
            if (lane == 0) {
                P.results[(size_t)et * P.num_envs + env] = 0;
                if (P.counters) atomicAdd(P.counters + 0, 1ull);
            }
            continue;
        }
        int bt = 0;
#pragma unroll
        for (int u = 0; u < SUB; ++u)
            if (u == t) bt = base[u];
        walk_listed_pair<M, MODE>(P, env, et, Cs[t], pairs + bt, prim, np, GL);
    }
    }
    __syncwarp();  // every lane is done with the lists before the next group's writes
}

// check_tile processes the edges of one (environment, edge tile) work item
// (modes 0 and 1) with the environment's records already staged in shared
// memory; it is shared by the one-CTA-per-item grid kernel and the persistent
// kernel.  Each warp takes pairs_per_setup consecutive edges at a time.
template <class M, int WARPS, int MODE>
__device__ __forceinline__ void check_tile(const CheckParams& P, int env, int tile, int n_slots,
                                           const unsigned char* smem, float4 h0, float4 h1,
                                           int* s_next = nullptr) {
    constexpr int SUB = pairs_per_setup<M>();
    const int e_begin = tile * P.edges_per_cta;
    const int warp = threadIdx.x >> 5;
    const uint32_t shape = __float_as_uint(h1.w);
    const int np = (int)(shape & 0xffffu);
    const int W = (int)(shape >> 16);  // 64-bit words per primitive mask
    const float4* prim = reinterpret_cast<const float4*>(smem);
    // the mask tables stay in global memory (read through L1): each pair reads
    // only the few words its slab ranges select
    const uint64_t* __restrict__ masks =
        reinterpret_cast<const uint64_t*>(P.blobs + (size_t)__float_as_uint(h0.w) + (size_t)np * kPrimF4);
    uint16_t* pairs =
        reinterpret_cast<uint16_t*>(const_cast<unsigned char*>(smem) + P.blob_smem) + (size_t)warp * P.pairs_per_warp;
    const GroupLanes GL = group_lanes<M>();
    if (s_next) {
        // Warps take the tile's next pass from a shared counter: a pass costs
        // from one chunk (a pair colliding at its first sample) to dozens (a
        // collision-free pair), so a fixed stride leaves warps idle while the
        // CTA's last one finishes.
        const int lane = threadIdx.x & 31;
        for (;;) {
            int slot = 0;
            if (lane == 0) slot = atomicAdd(s_next, SUB);
            slot = __shfl_sync(kFull, slot, 0);
            if (slot >= n_slots) break;
            if constexpr (SUB > 1)
                check_pair_group<M, MODE>(P, env, e_begin + slot, min(SUB, n_slots - slot), prim, masks, np, W,
                                          pairs, GL);
            else
                check_pair<M, MODE>(P, env, e_begin + slot, -1, prim, masks, np, W, pairs, nullptr, GL);
        }
    } else if constexpr (SUB > 1) {
        for (int slot = warp * SUB; slot < n_slots; slot += WARPS * SUB)
            check_pair_group<M, MODE>(P, env, e_begin + slot, min(SUB, n_slots - slot), prim, masks, np, W, pairs,
                                      GL);
    } else {
        for (int slot = warp; slot < n_slots; slot += WARPS)
            check_pair<M, MODE>(P, env, e_begin + slot, -1, prim, masks, np, W, pairs, nullptr, GL);
    }
}

__device__ __forceinline__ int tile_slots(const CheckParams& P, int tile) {
    const int e_begin = tile * P.edges_per_cta;
    return min(P.edges_per_cta, P.num_edges - e_begin);
}

// Bytes of an environment's primitive records (what a CTA stages).
__device__ __forceinline__ uint32_t record_bytes_of(float4 h1) {
    return (__float_as_uint(h1.w) & 0xffffu) * kPrimF4 * 16u;
}

// One CTA per (environment, edge tile): blockIdx.x = environment, blockIdx.y = tile.
// Check CTAs are compiled for M::check_warps_per_sm resident warps per SM (a
// register budget of 65536 / (32 x that) per thread), at most 32 CTAs per SM.
template <class M, int WARPS>
constexpr int check_min_ctas() {
    return M::check_warps_per_sm / WARPS < 32 ? M::check_warps_per_sm / WARPS : 32;
}

template <class M, int WARPS, int MODE>
__global__ void __launch_bounds__(WARPS * 32, check_min_ctas<M, WARPS>()) check_kernel(CheckParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ int s_next;
    const int env = blockIdx.x, tile = blockIdx.y;
    const int n_slots = tile_slots(P, tile);
    if (n_slots <= 0) return;
    const float4 h0 = P.env_hdr[2 * env + 0];
    const float4 h1 = P.env_hdr[2 * env + 1];
    const uint32_t bytes = record_bytes_of(h1);
    if (threadIdx.x == 0) s_next = 0;
    if (bytes) {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x == 0) bulk_copy_g2s(smem, P.blobs + (size_t)__float_as_uint(h0.w), bytes, &bar);
        // The whole CTA takes one path: if any thread gave up, all flag, wait once
        // more (bounded) for the copy in flight, and return together.
        const bool ok = mbar_wait_bounded(&bar, 0u, 1u << 22);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicOr(P.error_flag, 1);
            mbar_wait_bounded(&bar, 0u, 1u << 22);
            return;
        }
    } else {
        __syncthreads();  // s_next is set before any warp takes a pass
    }
    check_tile<M, WARPS, MODE>(P, env, tile, n_slots, smem, h0, h1, &s_next);
}

// Persistent: a grid sized to the resident capacity pulls environment-major
// work items (environment, edge tile) from an atomic counter, two at a time so
// that consecutive items usually share the environment and its staged blob.
constexpr int kItemsPerGrab = 2;

template <class M, int WARPS, int MODE>
__global__ void __launch_bounds__(WARPS * 32, check_min_ctas<M, WARPS>()) check_persistent_kernel(CheckParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ int s_item;
    __shared__ int s_next[kItemsPerGrab];  // per grabbed item: the next pass a warp takes
    const int tiles = (P.num_edges + P.edges_per_cta - 1) / P.edges_per_cta;
    const long long items = (long long)P.num_envs * tiles;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int staged = -1;
    uint32_t phase = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(P.work_counter, kItemsPerGrab);
            for (int i = 0; i < kItemsPerGrab; ++i) s_next[i] = 0;
        }
        __syncthreads();
        const int first = s_item;
        __syncthreads();
        if (first >= items) break;
        bool failed = false;
        for (int item = first; item < first + kItemsPerGrab && item < items; ++item) {
            const int env = item / tiles, tile = item - (item / tiles) * tiles;
            const int n_slots = tile_slots(P, tile);
            if (n_slots <= 0) continue;
            const float4 h0 = P.env_hdr[2 * env + 0];
            const float4 h1 = P.env_hdr[2 * env + 1];
            if (env != staged) {
                const uint32_t bytes = record_bytes_of(h1);
                __syncthreads();  // every warp is done with the previous blob
                if (bytes) {
                    if (threadIdx.x == 0) bulk_copy_g2s(smem, P.blobs + (size_t)__float_as_uint(h0.w), bytes, &bar);
                    const bool ok = mbar_wait_bounded(&bar, phase, 1u << 22);
                    if (__syncthreads_or(!ok)) {
                        if (threadIdx.x == 0) atomicOr(P.error_flag, 1);
                        mbar_wait_bounded(&bar, phase, 1u << 22);
                        failed = true;
                        break;
                    }
                    phase ^= 1u;
                }
                staged = env;
            }
            check_tile<M, WARPS, MODE>(P, env, tile, n_slots, smem, h0, h1, &s_next[item - first]);
        }
        if (failed) break;
        __syncthreads();
    }
}

// Learned order, phase 3: each CTA pulls queued pairs from finish_counter, one
// at a time, and its warps split each pair's walk (warp w takes chunks w,
// w + WARPS, ... of the learned order; a hit in any stops all): the queued
// pairs are the longest walks of the check, and one warp per pair would leave
// the slowest single walk as the kernel's critical path.  The verdict is the
// OR over all items, so the split changes no verdict.  Consecutive pulls
// belong to different environments, so the primitive records are read from
// global memory (L1/L2) rather than staged; shared memory holds the warps'
// pair lists only (each warp compacts its own copy).  Compiled for at most 32
// resident warps per SM: its walk holds 64-bit record pointers and the segment
// permutation, and spills in the plain check kernel's tighter register budget.
template <class M, int WARPS>
constexpr int finish_min_ctas() {
    return (M::check_warps_per_sm < 32 ? M::check_warps_per_sm : 32) / WARPS;
}

// Learned order, phase 3, one warp per queued pair: each warp pulls entries
// from finish_counter on its own, culls, ranks the segments and walks the
// pair in learned order (MODE 3).  No CTA barrier per pair, so many pairs are
// in flight per SM; a long walk is not split, so the longest queued pair sets
// the tail.  Compiled like finish_kernel.
template <class M, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, finish_min_ctas<M, WARPS>()) finish_warp_kernel(CheckParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint8_t s_perm[WARPS][kMaxSegments];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long queued = (long long)(*P.q_head >> 32);
    const int total = (int)min(queued, (long long)P.q_cap);
    uint16_t* pairs = reinterpret_cast<uint16_t*>(smem) + (size_t)warp * P.pairs_per_warp;
    const GroupLanes GL = group_lanes<M>();
    for (;;) {
        int i = 0;
        if (lane == 0) i = atomicAdd(P.finish_counter, 1);
        i = __shfl_sync(kFull, i, 0);
        if (i >= total) break;
        const int ro = P.q_rows[i];
        if (ro < 0) continue;  // the probe walked this pair on
        const int2 pe = P.q_pairs[i];
        const float4 h0 = P.env_hdr[2 * pe.y + 0];
        const float4 h1 = P.env_hdr[2 * pe.y + 1];
        const uint32_t shape = __float_as_uint(h1.w);
        const int np = (int)(shape & 0xffffu);
        const int W = (int)(shape >> 16);
        const float4* prim = P.blobs + __float_as_uint(h0.w);
        const uint64_t* masks = reinterpret_cast<const uint64_t*>(prim + (size_t)np * kPrimF4);
        check_pair<M, 3>(P, pe.y, pe.x, ro, prim, masks, np, W, pairs, s_perm[warp], GL);
    }
}

template <class M, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, finish_min_ctas<M, WARPS>()) finish_kernel(CheckParams P) {
    constexpr int G = M::num_env_groups;
    constexpr int GB = group_bits<M>();
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint8_t s_perm[WARPS][kMaxSegments];
    __shared__ int s_item, s_C;
    __shared__ volatile int s_hit;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long queued = (long long)(*P.q_head >> 32);
    const int total = (int)min(queued, (long long)P.q_cap);
    // Warp 0 culls and compacts each pair once into the CTA's list (all the
    // warps' buffers together); a pair whose list would not fit falls back to
    // per-warp lists (each warp its own copy, walked in segments).
    uint16_t* cta_pairs = reinterpret_cast<uint16_t*>(smem);
    const int cta_cap = WARPS * P.pairs_per_warp;
    uint16_t* pairs = cta_pairs + (size_t)warp * P.pairs_per_warp;
    const GroupLanes GL = group_lanes<M>();
    for (;;) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(P.finish_counter, 1);
            s_hit = 0;
        }
        __syncthreads();
        const int i = s_item;
        if (i >= total) break;  // CTA-uniform
        const int ro = P.q_rows[i];
        const int2 pe = ro >= 0 ? P.q_pairs[i] : make_int2(0, 0);
        if (ro >= 0) {  // ro < 0: the probe walked this pair on
            const int env = pe.y, e = pe.x;
            const float4 h0 = P.env_hdr[2 * env + 0];
            const float4 h1 = P.env_hdr[2 * env + 1];
            const uint32_t shape = __float_as_uint(h1.w);
            const int np = (int)(shape & 0xffffu);
            const int W = (int)(shape >> 16);
            const float4* prim = P.blobs + __float_as_uint(h0.w);
            const uint64_t* masks = reinterpret_cast<const uint64_t*>(prim + (size_t)np * kPrimF4);
            const int n = P.steps[e];
            const int nseg = 4 * n;
            if (warp == 0) {
                // A queued pair passed the probe's self-collision test and has
                // candidates; the cull below repeats the probe's exactly.
                const int code = lane < G ? P.edge_tri[(size_t)e * G + lane] : -1;
                auto mask_word = [&](int w) {
                    const int tx = code & 1023, ty = (code >> 10) & 1023, tz = code >> 20;
                    return __ldg(masks + tx * W + w) & __ldg(masks + (kGridTri + ty) * W + w) &
                           __ldg(masks + (2 * kGridTri + tz) * W + w);
                };
                int cnt = 0;
                if (code >= 0 && np > 0)
                    for (int w = 0; w < W; ++w) cnt += __popcll(mask_word(w));
                int off = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(kFull, off, o);
                    if (lane >= o) off += y;
                }
                const int C = __shfl_sync(kFull, off, 31);
                off -= cnt;
                const bool fits = C <= cta_cap && nseg <= kMaxSegments;
                if (fits && cnt > 0) {
                    int idx = off;
                    for (int w = 0; w < W; ++w) {
                        uint64_t m = mask_word(w);
                        while (m) {
                            const int b = __ffsll((long long)m) - 1;
                            cta_pairs[idx++] = (uint16_t)(((w * 64 + b) << GB) | lane);
                            m &= m - 1;
                        }
                    }
                }
                if (fits) learned_perm(P, ro, nseg, s_perm[0]);
                if (lane == 0) {
                    s_C = fits ? C : -1;
                    if (fits && P.counters) atomicAdd(P.counters + 1, (unsigned long long)C);
                }
            }
            __syncthreads();
            const int C = s_C;
            if (C > 0) {
                bool undecided = false;
                WalkStats st;
                walk_pairs<M, 2>(P.table, (size_t)P.offs[e], n, C, cta_pairs, prim, np, s_perm[0], 0, GL, undecided,
                                 st, [] { return false; }, 32 * warp, -1, WARPS, &s_hit);
                if (lane == 0 && P.counters) {
                    atomicAdd(P.counters + 2, (unsigned long long)st.chunks);
                    atomicAdd(P.counters + 3, (unsigned long long)st.gates);
                    atomicAdd(P.counters + 4, (unsigned long long)st.leaf);
                }
            } else if (C < 0) {
                check_pair<M, 2>(P, env, e, ro, prim, masks, np, W, pairs, s_perm[warp], GL, warp, WARPS, &s_hit);
            }
        }
        __syncthreads();  // every warp is done with this pair (and with s_item)
        if (threadIdx.x == 0 && ro >= 0) {
            P.results[(size_t)pe.x * P.num_envs + pe.y] = s_hit ? 1 : 0;
            if (P.counters) {
                atomicAdd(P.counters + 0, 1ull);
                atomicAdd(P.counters + 5, s_hit ? 1ull : 0ull);
            }
        }
    }
}

// ------------------------------------------------------------------ learned order
// One MLP feature row: joints normalised to [-1, 1] by the joint limits, the
// environment code, zeros, and in column kMlpIn - 2 the sample's position
// along its edge (sample k of 32 n mapped to [-1, 1]: where on an edge whose
// start is free a collision lies is the strongest per-sample signal the
// walk order can use); column kMlpIn - 1 stays zero (the forward kernel's bias
// input).  BF16, kMlpIn values.
__device__ __forceinline__ float sample_position(int k, int n) {
    return 2.0f * (float)k / (float)(kLanes * n - 1) - 1.0f;
}

template <class M>
__device__ __forceinline__ void write_features(const float* q, const float* code, float pos, uint16_t* dst) {
    static_assert(M::dof + kEnvCode <= kMlpIn - 2, "feature row too narrow for this robot");
    const DevTables<M>& T = tab<M>();
    float f[kMlpIn];
#pragma unroll
    for (int j = 0; j < kMlpIn; ++j) f[j] = 0.0f;
#pragma unroll
    for (int j = 0; j < M::dof; ++j) f[j] = 2.0f * (q[j] - T.s_a[j]) / T.s_m[j] - 1.0f;
#pragma unroll
    for (int j = 0; j < kEnvCode; ++j) f[M::dof + j] = code[j];
    f[kMlpIn - 2] = pos;
    uint32_t w[kMlpIn / 2];
#pragma unroll
    for (int j = 0; j < kMlpIn / 2; ++j) {
        __nv_bfloat162 h = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
        w[j] = *reinterpret_cast<uint32_t*>(&h);
    }
    uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
    for (int j = 0; j < kMlpIn / 8; ++j) d[j] = make_uint4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
}

// Features of every queued pair's segments: row ro + j is segment j scored at
// its last sample k = 8 j + 7, the first one the finish walk checks.  Eight
// lanes per queue entry (four entries per
// warp in flight, grid-strided), each lane one segment at a time: the loads
// of an entry form a dependent chain, so several entries per warp hide it.
constexpr int kFeatureLanes = 8;

template <class M>
__global__ void queue_features_kernel(CheckParams P, const float* __restrict__ edges, const float* __restrict__ code,
                                      uint16_t* __restrict__ x) {
    const int sl = threadIdx.x & (kFeatureLanes - 1);
    const long long queued = (long long)(*P.q_head >> 32);
    const int total = (int)min(queued, (long long)P.q_cap);
    const int per_cta = blockDim.x / kFeatureLanes;
    const int stride = gridDim.x * per_cta;
    for (int i = blockIdx.x * per_cta + threadIdx.x / kFeatureLanes; i < total; i += stride) {
        const int ro = P.q_rows[i];
        if (ro < 0) continue;
        const int2 pe = P.q_pairs[i];
        const int e = pe.x, env = pe.y;
        const int n = P.steps[e];
        float s[M::dof], t[M::dof], q[M::dof];
#pragma unroll
        for (int j = 0; j < M::dof; ++j) {
            s[j] = edges[(size_t)e * 2 * M::dof + j];
            t[j] = edges[(size_t)e * 2 * M::dof + M::dof + j];
        }
        for (int seg = sl; seg < 4 * n; seg += kFeatureLanes) {
            const int k = seg * kSegment + kSegment - 1;
            edge_sample<M::dof>(s, t, n, k, q);
            write_features<M>(q, code + (size_t)env * kEnvCode, sample_position(k, n), x + (size_t)(ro + seg) * kMlpIn);
        }
    }
}

// Inline learned order, features: row c * S + s (S = the check's segments,
// offs[E] / 8) is segment s of its edge scored at its last sample with the
// code of environment cluster c.  One thread per row.
template <class M>
__global__ void cluster_features_kernel(CheckParams P, const float* __restrict__ edges,
                                        const float* __restrict__ centroids, int K, const int* __restrict__ row_edge,
                                        uint16_t* __restrict__ x) {
    const long long S = P.total_segs;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S * K) return;
    const int c = (int)(i / S);
    const int sg = (int)(i - (long long)c * S);
    // the segment's edge: segments never straddle edges (offs[e] % 32 == 0);
    // binary search over the sample offsets (the FK table may not exist yet)
    const int row = sg * kSegment;
    int lo = 0, hi = P.num_edges - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.offs[mid] <= row) lo = mid; else hi = mid - 1;
    }
    const int e = lo;
    (void)row_edge;
    const int j = sg - P.offs[e] / kSegment;
    float s[M::dof], t[M::dof], q[M::dof];
#pragma unroll
    for (int d = 0; d < M::dof; ++d) {
        s[d] = edges[(size_t)e * 2 * M::dof + d];
        t[d] = edges[(size_t)e * 2 * M::dof + M::dof + d];
    }
    const int k = j * kSegment + kSegment - 1;
    edge_sample<M::dof>(s, t, P.steps[e], k, q);
    write_features<M>(q, centroids + (size_t)c * kEnvCode, sample_position(k, P.steps[e]), x + (size_t)i * kMlpIn);
}

// Inline learned order, permutations: one warp per (cluster c, edge e).
// Lane block t is scored by the segment holding its last sample t n + n - 1
// (row c * S + offs[e] / 8 + segment); blocks are ranked by descending score,
// ties (blocks of one segment) by descending index, so a segment is walked
// from its end back, and block 0 is ranked first.  perms[(c * E + e) * 32 +
// rank] = block.
template <class M>
__global__ void cluster_perm_kernel(CheckParams P, int K, uint8_t* __restrict__ perms) {
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int E = P.num_edges;
    if (warp >= (long long)K * E) return;
    const int c = (int)(warp / E);
    const int e = (int)(warp - (long long)c * E);
    const int n = P.steps[e];
    float v = P.logits[(size_t)c * P.total_segs + P.offs[e] / kSegment + (lane * n + n - 1) / kSegment];
    v = isnan(v) ? -INFINITY : v;
    if (lane == 0) v = INFINITY;
    int rank = 0;
    for (int u = 0; u < kLanes; ++u) {
        const float vu = __shfl_sync(kFull, v, u);
        rank += (vu > v || (vu == v && u > lane)) ? 1 : 0;
    }
    perms[((size_t)c * E + e) * kLanes + rank] = (uint8_t)lane;
}

// Training rows: row i draws (environment, edge, sample) from a hash of
// (seed, i); features as above at that sample; label = the sample's
// environment collision with the reference's gate semantics (bound against
// every primitive, then the leaves against every primitive).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Environment verdict of one sample-table row against environment env, one
// thread: each link group's bound against every primitive and, once some
// primitive hits it, the group's leaves against every primitive -- the
// reference's gate semantics (fkcc, src/utils.cuh:806-1190).  Self-collision
// is not part of it (env-independent, decided per edge before any walk).
template <class M>
__device__ __forceinline__ bool sample_hits_env(const CheckParams& P, int env, size_t row) {
    constexpr int G = M::num_env_groups;
    const float4 hd0 = P.env_hdr[2 * env], hd1 = P.env_hdr[2 * env + 1];
    const float4* rec = P.blobs + __float_as_uint(hd0.w);
    const int np = (int)(__float_as_uint(hd1.w) & 0xffffu);
    const float4* r = P.table + table_index<M>(row, 0);  // sphere s at r[s * M::table_tile]
    const DevTables<M>& T = tab<M>();
    for (int g = 0; g < G; ++g) {
        float4 b = r[g * M::table_tile];
        b.w += kEnvInflate;
        bool gate = false;
        for (int p = 0; p < np && !gate; ++p) gate = sphere_hits_prim(b, rec + p * kPrimF4);
        if (!gate) continue;
        for (int li = T.leaf_begin[g]; li < T.leaf_begin[g + 1]; ++li) {
            float4 l = r[(G + li) * M::table_tile];
            l.w += kEnvInflate;
            for (int p = 0; p < np; ++p)
                if (sphere_hits_prim(l, rec + p * kPrimF4)) return true;
        }
    }
    return false;
}

// Learned-order population: the environment verdict of every sample of every
// queued pair (one warp per queue entry, lanes over the 32 n samples):
// lab[8 ro + k] for sample k of the entry whose first MLP row is ro, and
// y[ro + j] = the verdict at segment j's scored sample 8 j + 7.
template <class M>
__global__ void queue_labels_kernel(CheckParams P, uint8_t* __restrict__ lab, uint8_t* __restrict__ y) {
    const int lane = threadIdx.x & 31;
    const long long queued = (long long)(*P.q_head >> 32);
    const int total = (int)min(queued, (long long)P.q_cap);
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        const int ro = P.q_rows[i];
        if (ro < 0) continue;
        const int2 pe = P.q_pairs[i];
        const int n = P.steps[pe.x];
        const size_t row0 = (size_t)P.offs[pe.x];
        for (int k = lane; k < kLanes * n; k += 32) {
            const uint8_t h = sample_hits_env<M>(P, pe.y, row0 + (size_t)k) ? 1 : 0;
            lab[(size_t)ro * kSegment + k] = h;
            if ((k & (kSegment - 1)) == kSegment - 1) y[ro + k / kSegment] = h;
        }
    }
}

template <class M>
__global__ void training_rows_kernel(CheckParams P, const float* __restrict__ edges, const float* __restrict__ code,
                                     long long rows, unsigned long long seed, uint16_t* __restrict__ x,
                                     uint8_t* __restrict__ y) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const unsigned long long h1 = mix64(seed ^ (unsigned long long)i), h2 = mix64(h1), h3 = mix64(h2);
    const int env = (int)(h1 % (unsigned long long)P.num_envs);
    const int e = (int)(h2 % (unsigned long long)P.num_edges);
    const int n = P.steps[e];
    const int k = (int)(h3 % (unsigned long long)(kLanes * n));
    float s[M::dof], t[M::dof], q[M::dof];
#pragma unroll
    for (int j = 0; j < M::dof; ++j) {
        s[j] = edges[(size_t)e * 2 * M::dof + j];
        t[j] = edges[(size_t)e * 2 * M::dof + M::dof + j];
    }
    edge_sample<M::dof>(s, t, n, k, q);
    write_features<M>(q, code + (size_t)env * kEnvCode, sample_position(k, n), x + (size_t)i * kMlpIn);
    y[i] = sample_hits_env<M>(P, env, (size_t)P.offs[e] + k) ? 1 : 0;
}

// ------------------------------------------------------------------ records variant
// Environment check from the host-packed rounded-box records of bcc_pack_envs
// (no interval-mask tables), used by the allocation-free entry point: culls
// (primitive, link) pairs with an exact AABB overlap test, one primitive per
// lane; the walk over (sample, pair) items is check_kernel's.
template <class M, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) check_records_kernel(RecordsParams P) {
    constexpr int G = M::num_env_groups;
    constexpr int GB = group_bits<M>();
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ float4 boxes[WARPS][G][2];

    const int env = blockIdx.x;
    const int e_begin = blockIdx.y * P.edges_per_cta;
    const int e_end = min(e_begin + P.edges_per_cta, P.num_edges);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p_begin = P.env_off[env];
    const int np = P.env_off[env + 1] - p_begin;

    const float4* prim = reinterpret_cast<const float4*>(smem);
    uint16_t* pairs = reinterpret_cast<uint16_t*>(smem + (size_t)P.max_prims * kPrimF4 * 16) +
                      (size_t)warp * P.pairs_per_warp;
    if (np < 0 || np > P.max_prims) {  // shared memory was sized from the caller's max_prims
        if (threadIdx.x == 0) atomicOr(P.error_flag, 2);
        return;
    }
    if (np > 0) {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x == 0)
            bulk_copy_g2s(smem, P.records + (size_t)p_begin * kPrimF4, (uint32_t)np * kPrimF4 * 16u, &bar);
        // One path for the whole CTA (see check_kernel).
        const bool ok = mbar_wait_bounded(&bar, 0u, 1u << 22);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicOr(P.error_flag, 1);
            mbar_wait_bounded(&bar, 0u, 1u << 22);
            return;
        }
    }
    const uint32_t lt = (1u << lane) - 1u;
    const GroupLanes GL = group_lanes<M>();

    for (int e = e_begin + warp; e < e_end; e += WARPS) {
        uint8_t* out = P.results + (size_t)e * P.num_envs + env;
        const int self = P.edge_self[e];
        if (np == 0 || self) {
            if (lane == 0) *out = self ? 1 : 0;
            continue;
        }
        if (lane < G) {
            boxes[warp][lane][0] = P.swept[((size_t)e * G + lane) * 2 + 0];
            boxes[warp][lane][1] = P.swept[((size_t)e * G + lane) * 2 + 1];
        }
        __syncwarp();
        // Exact AABB cull, one primitive per lane; pairs compacted link-major
        // within each block of 32 primitives.
        int C = 0;
        for (int p0 = 0; p0 < np; p0 += 32) {
            const int p = p0 + lane;
            uint32_t mask = 0;
            if (p < np) {
                const float4 c = prim[p * kPrimF4 + 0];
                const float4 h = prim[p * kPrimF4 + 4];
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    const float4 lo = boxes[warp][g][0], hi = boxes[warp][g][1];
                    const bool ov = c.x - h.x <= hi.x && c.x + h.x >= lo.x && c.y - h.y <= hi.y &&
                                    c.y + h.y >= lo.y && c.z - h.z <= hi.z && c.z + h.z >= lo.z;
                    mask |= (uint32_t)ov << g;
                }
            }
#pragma unroll 1
            for (int g = 0; g < G; ++g) {
                const uint32_t bits = __ballot_sync(kFull, (mask >> g) & 1u);
                if ((mask >> g) & 1u) pairs[C + __popc(bits & lt)] = (uint16_t)((p << GB) | g);
                C += __popc(bits);
            }
        }
        __syncwarp();

        bool collide = false, undecided = false;
        WalkStats st;
        if (C > 0)
            collide = walk_pairs<M, 0>(P.table, (size_t)P.offs[e], P.steps[e], C, pairs, prim, np, nullptr, 0,
                                       GL, undecided, st, [] { return false; });
        __syncwarp();
        if (lane == 0) *out = collide ? 1 : 0;
    }
}

// ------------------------------------------------------------------ launchers
template <class M>
cudaError_t run_steps(const PipelineArgs& a, cudaStream_t st) {
    const int E = a.num_edges;
    if (a.stage_events) cudaEventRecord(a.stage_events[0], st);
    edge_steps_kernel<M><<<(E + 255) / 256, 256, 0, st>>>(a.d_edges, E, a.resolution, a.steps);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    return launch_scan(a.steps, E, a.offs, st);
}

template <class M, int W, int MODE>
cudaError_t launch_check_wm(CheckParams P, int E, cudaStream_t st) {
    P.pairs_per_warp = std::min((P.max_prims * M::num_env_groups + 7) & ~7, kPairCap);
    const size_t smem = P.blob_smem + (size_t)W * P.pairs_per_warp * sizeof(uint16_t);
    if (P.persistent) {
        cudaError_t err = cudaFuncSetAttribute(check_persistent_kernel<M, W, MODE>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        int per_sm = 0, dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, check_persistent_kernel<M, W, MODE>, W * 32, smem);
        if (err != cudaSuccess) return err;
        const long long items = (long long)P.num_envs * ((E + P.edges_per_cta - 1) / P.edges_per_cta);
        long long grid = (long long)std::max(per_sm, 1) * std::max(sms, 1);
        grid = std::min(grid, (items + kItemsPerGrab - 1) / kItemsPerGrab);
        err = cudaMemsetAsync(P.work_counter, 0, sizeof(int), st);
        if (err != cudaSuccess) return err;
        check_persistent_kernel<M, W, MODE><<<(unsigned)std::max(grid, 1ll), W * 32, smem, st>>>(P);
        return cudaGetLastError();
    }
    cudaError_t err = cudaFuncSetAttribute(check_kernel<M, W, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
    if (err != cudaSuccess) return err;
    dim3 grid(P.num_envs, (E + P.edges_per_cta - 1) / P.edges_per_cta);
    check_kernel<M, W, MODE><<<grid, W * 32, smem, st>>>(P);
    return cudaGetLastError();
}

// Learned order, phase 3: a grid of the resident capacity; the queue length
// is read on the device.
template <class M, int W>
cudaError_t launch_finish_w(CheckParams P, cudaStream_t st) {
    P.pairs_per_warp = std::min((P.max_prims * M::num_env_groups + 7) & ~7, kPairCap);
    const size_t smem = (size_t)W * P.pairs_per_warp * sizeof(uint16_t);
    auto kern = P.finish_split ? finish_kernel<M, W> : finish_warp_kernel<M, W>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, W * 32, smem);
    if (err != cudaSuccess) return err;
    err = cudaMemsetAsync(P.finish_counter, 0, sizeof(int), st);
    if (err != cudaSuccess) return err;
    kern<<<std::max(per_sm, 1) * std::max(sms, 1), W * 32, smem, st>>>(P);
    return cudaGetLastError();
}

template <class M, int W>
cudaError_t launch_check_w(CheckParams P, int E, cudaStream_t st, int mode) {
    switch (mode) {
        case 1: return launch_check_wm<M, W, 1>(P, E, st);
        case 2: return launch_finish_w<M, W>(P, st);
        case 4: return launch_check_wm<M, W, 4>(P, E, st);
        case 5:  // 16 lanes per walking pair, where the robot has a grouped cull and no overhang
            if constexpr (!has_overhang<M>() && pairs_per_setup<M>() > 1) return launch_check_wm<M, W, 5>(P, E, st);
            return launch_check_wm<M, W, 0>(P, E, st);
        default: return launch_check_wm<M, W, 0>(P, E, st);
    }
}

template <class M>
cudaError_t check_by_warps(const CheckParams& P, int E, int warps, int mode, cudaStream_t st) {
    switch (warps) {
        case 8: return launch_check_w<M, 8>(P, E, st, mode);
        case 4: return launch_check_w<M, 4>(P, E, st, mode);
        case 2: return launch_check_w<M, 2>(P, E, st, mode);
        case 1: return launch_check_w<M, 1>(P, E, st, mode);
        default: return cudaErrorInvalidValue;
    }
}

// FK table, self-collision and swept volumes (no environment check); records
// stage events 1-4 when profiling.
template <class M>
cudaError_t run_prep(const PipelineArgs& a, cudaStream_t st) {
    const int E = a.num_edges;
    const int R = a.total_rows;
    cudaEvent_t* ev = a.stage_events;
    if (ev) cudaEventRecord(ev[1], st);
    cudaError_t err = cudaMemsetAsync(a.edge_self, 0, sizeof(int) * E, st);
    if (err != cudaSuccess) return err;
    if (R > 0) {
        if constexpr (M::table_tile == 1) {
            // FK and self-collision in one kernel; a grid of the resident CTAs
            // strides over the 32-row blocks
            const size_t smem = 32 * (size_t)(M::num_spheres | 1) * sizeof(float4);
            err = cudaFuncSetAttribute(fk_staged_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (err != cudaSuccess) return err;
            int dev = 0, sms = 0, per_sm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fk_staged_kernel<M>, 32, smem);
            if (err != cudaSuccess) return err;
            const int blocks = (R + 31) / 32;
            const int grid = std::min(blocks, std::max(per_sm, 1) * std::max(sms, 1));
            fk_staged_kernel<M><<<grid, 32, smem, st>>>(a.d_edges, E, a.steps, a.offs, a.table, a.row_edge, a.fk_perm,
                                                        a.edge_self);
        } else {
            fk_kernel<M><<<(R + 127) / 128, 128, 0, st>>>(a.d_edges, E, a.steps, a.offs, a.table, a.row_edge,
                                                           a.fk_perm);
        }
    }
    if (ev) cudaEventRecord(ev[2], st);
    if constexpr (M::table_tile != 1) {  // row-major tables: checked by fk_staged_kernel
        if (R > 0) {
            // one warp per row; a grid of at most 16 CTAs per SM strides over the rows
            int dev = 0, sms = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            const long long want = ((long long)R * 32 + kSelfThreads - 1) / kSelfThreads;
            const int grid = (int)std::min<long long>(want, 16ll * std::max(sms, 1));
            self_kernel<M><<<grid, kSelfThreads, 0, st>>>(a.table, R, a.row_edge, a.edge_self);
        }
    }
    if (ev) cudaEventRecord(ev[3], st);
    swept_kernel<M><<<(E * 32 + 255) / 256, 256, 0, st>>>(a.table, a.offs, E, a.swept,
                                                           a.grid_bounds ? a.edge_tri : nullptr, a.grid_bounds);
    if (ev) cudaEventRecord(ev[4], st);
    return cudaGetLastError();
}

// Environment check only (the FK/self/swept stages already ran), in a.mode.
template <class M>
cudaError_t run_check_mode(const PipelineArgs& a, cudaStream_t st) {
    return check_by_warps<M>(params_of(a), a.num_edges, a.warps, a.mode, st);
}

template <class M>
cudaError_t run_check(const PipelineArgs& a, cudaStream_t st) {
    cudaError_t err = run_prep<M>(a, st);
    if (err != cudaSuccess) return err;
    err = run_check_mode<M>(a, st);
    if (a.stage_events) cudaEventRecord(a.stage_events[5], st);
    return err;
}

template <class M>
cudaError_t run_queue_features(const PipelineArgs& a, const float* env_code, uint16_t* x, int grid,
                               cudaStream_t st) {
    if (grid <= 0) return cudaSuccess;
    queue_features_kernel<M><<<grid, 128, 0, st>>>(params_of(a), a.d_edges, env_code, x);
    return cudaGetLastError();
}

template <class M>
cudaError_t run_cluster_order_inputs(const PipelineArgs& a, const float* centroids, int K, uint16_t* x,
                                     cudaStream_t st) {
    const long long rows = (long long)K * a.total_segs;
    if (rows <= 0) return cudaSuccess;
    cluster_features_kernel<M><<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(params_of(a), a.d_edges, centroids, K,
                                                                               a.row_edge, x);
    return cudaGetLastError();
}

template <class M>
cudaError_t run_cluster_perms(const PipelineArgs& a, int K, uint8_t* perms, cudaStream_t st) {
    const long long warps = (long long)K * a.num_edges;
    if (warps <= 0) return cudaSuccess;
    cluster_perm_kernel<M><<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(params_of(a), K, perms);
    return cudaGetLastError();
}

template <class M>
cudaError_t run_training_rows(const PipelineArgs& a, const float* env_code, long long rows, unsigned long long seed,
                              uint16_t* x, uint8_t* y, cudaStream_t st) {
    if (rows <= 0) return cudaSuccess;
    training_rows_kernel<M><<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(params_of(a), a.d_edges, env_code, rows,
                                                                           seed, x, y);
    return cudaGetLastError();
}

template <class M>
cudaError_t run_queue_labels(const PipelineArgs& a, uint8_t* lab, uint8_t* y, int grid, cudaStream_t st) {
    if (grid <= 0) return cudaSuccess;
    queue_labels_kernel<M><<<grid, 256, 0, st>>>(params_of(a), lab, y);
    return cudaGetLastError();
}

template <class M>
cudaError_t run_check_records(RecordsParams P, cudaStream_t st) {
    constexpr int W = kRecordsWarps;
    if (P.max_prims > max_prims_of<M>()) return cudaErrorInvalidValue;
    P.pairs_per_warp = (P.max_prims * M::num_env_groups + 7) & ~7;
    const size_t smem = records_smem_bytes(P.max_prims, M::num_env_groups, W);
    cudaError_t err = cudaFuncSetAttribute(check_records_kernel<M, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
    if (err != cudaSuccess) return err;
    dim3 grid(P.num_envs, (P.num_edges + P.edges_per_cta - 1) / P.edges_per_cta);
    check_records_kernel<M, W><<<grid, W * 32, smem, st>>>(P);
    return cudaGetLastError();
}

// The robot's entry points, as the robot-independent code calls them.
template <class M>
RobotOps robot_ops_of(int robot, cudaError_t (*upload)()) {
    RobotOps o;
    o.robot = robot;
    o.dof = M::dof;
    o.num_spheres = M::num_spheres;
    o.num_env_groups = M::num_env_groups;
    o.max_prims = max_prims_of<M>();
    o.half_warp_walk = !has_overhang<M>() && pairs_per_setup<M>() > 1;
    o.upload_tables = upload;
    o.steps = run_steps<M>;
    o.check = run_check<M>;
    o.prep = run_prep<M>;
    o.check_mode = run_check_mode<M>;
    o.queue_features = run_queue_features<M>;
    o.training_rows = run_training_rows<M>;
    o.queue_labels = run_queue_labels<M>;
    o.cluster_features = run_cluster_order_inputs<M>;
    o.cluster_perms = run_cluster_perms<M>;
    o.check_records = run_check_records<M>;
    return o;
}

}  // namespace bcc
