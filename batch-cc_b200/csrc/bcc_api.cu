// bcc_api.cu -- C ABI of the checker (include/bcc.h): context, environment
// arena upload, and the check entry points.
//
// Replaces the reference host entry batch_cc::batch_cc<Robot>
// (src/batch_cc.cu:244-338): instead of two cudaMalloc + a pinned staging blob
// per environment and a device pointer table, all environments live in one
// packed arena of 80-byte rounded-box records that persists across calls; the
// per-call buffers (edges, sample table, verdicts) are grown on demand and
// reused.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/bcc.h"
#include "bcc_device.cuh"
#include "bcc_kernels.h"
#include "bcc_mlp.h"

#include "bcc_ctx.h"

namespace {

bcc_status fail(bcc_ctx* c, bcc_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}

bcc_status cuda_fail(bcc_ctx* c, cudaError_t e, const char* what) {
    return fail(c, BCC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BCC_CUDA(ctx, call)                                          \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return cuda_fail((ctx), _e, #call);   \
    } while (0)

// Orthonormal pair completing unit vector a (FP64).
void complete_basis(const double a[3], double u[3], double w[3]) {
    double t[3] = {0, 0, 0};
    int m = std::fabs(a[0]) <= std::fabs(a[1]) ? (std::fabs(a[0]) <= std::fabs(a[2]) ? 0 : 2)
                                               : (std::fabs(a[1]) <= std::fabs(a[2]) ? 1 : 2);
    t[m] = 1.0;
    double d = t[0] * a[0] + t[1] * a[1] + t[2] * a[2];
    for (int i = 0; i < 3; ++i) u[i] = t[i] - d * a[i];
    double nu = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    for (int i = 0; i < 3; ++i) u[i] /= nu;
    w[0] = a[1] * u[2] - a[2] * u[1];
    w[1] = a[2] * u[0] - a[0] * u[2];
    w[2] = a[0] * u[1] - a[1] * u[0];
}

struct Rec {
    float v[20];
};

// Rounded box: centre c, axes A (rows), half-extents h, rounding radius rho.
Rec make_rec(const double c[3], const double A[3][3], const double h[3], double rho) {
    Rec r;
    r.v[0] = (float)c[0];
    r.v[1] = (float)c[1];
    r.v[2] = (float)c[2];
    r.v[3] = (float)rho;
    for (int i = 0; i < 3; ++i) {
        r.v[4 + 4 * i + 0] = (float)A[i][0];
        r.v[4 + 4 * i + 1] = (float)A[i][1];
        r.v[4 + 4 * i + 2] = (float)A[i][2];
        r.v[4 + 4 * i + 3] = (float)h[i];
    }
    // AABB half-size of the rounded box (+ cull margin), rounded outward.
    for (int k = 0; k < 3; ++k) {
        double hs = rho;
        for (int i = 0; i < 3; ++i) hs += std::fabs((double)(float)A[i][k]) * h[i];
        hs = hs * (1.0 + 1e-6) + 1e-6 + (double)bcc::kCullMargin;
        r.v[16 + k] = (float)hs;
    }
    r.v[19] = 0.0f;
    return r;
}

Rec rec_sphere(const float* s) {
    double c[3] = {s[0], s[1], s[2]};
    double A[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    double h[3] = {0, 0, 0};
    return make_rec(c, A, h, s[3]);
}

// Capsule x1 y1 z1 xv yv zv r rdv: segment p1 -> p1 + v with radius r
// (src/utils.cuh:114-127).  A zero-length segment is the sphere at p1, which is
// what the reference's NaN clamp (rdv = inf) evaluates to.
Rec rec_capsule(const float* k, bool z_aligned) {
    double p1[3] = {k[0], k[1], k[2]};
    double v[3] = {z_aligned ? 0.0 : (double)k[3], z_aligned ? 0.0 : (double)k[4], (double)k[5]};
    double L = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double c[3], A[3][3], h[3] = {0, 0, 0};
    double a[3] = {0, 0, 1};
    if (L > 0) {
        for (int i = 0; i < 3; ++i) a[i] = v[i] / L;
        h[2] = 0.5 * L;
    }
    for (int i = 0; i < 3; ++i) c[i] = p1[i] + 0.5 * v[i];
    double u[3], w[3];
    complete_basis(a, u, w);
    for (int i = 0; i < 3; ++i) {
        A[0][i] = u[i];
        A[1][i] = w[i];
        A[2][i] = a[i];
    }
    return make_rec(c, A, h, k[6]);
}

// Cuboid x y z a1 a2 a3 h1 h2 h3 (src/utils.cuh:159-178); the z-aligned variant
// projects on (a1x, a1y, 0), (a2x, a2y, 0) and (0, 0, 1) (:187-205).
Rec rec_cuboid(const float* b, bool z_aligned) {
    double c[3] = {b[0], b[1], b[2]};
    double A[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[i][j] = b[3 + 3 * i + j];
    if (z_aligned) {
        A[0][2] = 0;
        A[1][2] = 0;
        A[2][0] = 0;
        A[2][1] = 0;
        A[2][2] = 1;
    }
    double h[3] = {b[12], b[13], b[14]};
    return make_rec(c, A, h, 0.0);
}

int clamp_tile(int v, int lo, int hi) { return std::max(lo, std::min(hi, v)); }

// Discretisation, sample offsets and every per-call buffer of a check; fills
// `a` up to (not including) the FK / self / swept / check launches.
bcc_status prepare(bcc_ctx* ctx, bcc_robot robot, const float* d_edges, int E, int resolution, uint8_t* d_results,
                   const bcc_opts* opts, cudaStream_t st, bcc::PipelineArgs& a) {
    const int r = (int)robot;
    const bcc::RobotOps* ops = bcc::robot_ops(r);
    if (!ops) return fail(ctx, BCC_ERR_NOT_SUPPORTED, "robot not built into this library");
    if (ctx->max_prims > ops->max_prims)
        return fail(ctx, BCC_ERR_LIMIT, "an environment has more primitives than this robot's checker supports");
    if (!ctx->tables[r]) {
        BCC_CUDA(ctx, ops->upload_tables());
        ctx->tables[r] = true;
    }
    a = bcc::PipelineArgs{};
    a.d_edges = d_edges;
    a.num_edges = E;
    a.resolution = resolution;
    BCC_CUDA(ctx, ctx->steps.ensure(sizeof(int) * (size_t)E));
    BCC_CUDA(ctx, ctx->offs.ensure(sizeof(int) * ((size_t)E + 1)));
    BCC_CUDA(ctx, ctx->edge_self.ensure(sizeof(int) * (size_t)E));
    const int G = ops->num_env_groups;
    BCC_CUDA(ctx, ctx->swept.ensure(sizeof(float4) * 2 * (size_t)G * E));
    BCC_CUDA(ctx, ctx->edge_tri.ensure(sizeof(int) * (size_t)G * E));
    BCC_CUDA(ctx, ctx->error_flag.ensure(sizeof(int)));
    a.steps = ctx->steps.as<int>();
    a.offs = ctx->offs.as<int>();
    a.edge_self = ctx->edge_self.as<int>();
    a.swept = ctx->swept.as<float4>();
    a.edge_tri = ctx->edge_tri.as<int>();
    a.grid_bounds = ctx->grid_bounds.as<float>();
    a.error_flag = ctx->error_flag.as<int>();
    a.stage_events = ctx->profiling ? ctx->ev : nullptr;
    a.counters = nullptr;
    if (ctx->counting) {
        BCC_CUDA(ctx, ctx->counters.ensure(sizeof(unsigned long long) * bcc::kNumCounters));
        a.counters = ctx->counters.as<unsigned long long>();
        BCC_CUDA(ctx, cudaMemsetAsync(a.counters, 0, sizeof(unsigned long long) * bcc::kNumCounters, st));
    }
    BCC_CUDA(ctx, cudaMemsetAsync(a.error_flag, 0, sizeof(int), st));
    BCC_CUDA(ctx, ops->steps(a, st));
    BCC_CUDA(ctx, cudaMemcpyAsync(ctx->h_total, a.offs + E, sizeof(int), cudaMemcpyDeviceToHost, st));
    BCC_CUDA(ctx, cudaStreamSynchronize(st));
    const int total = *ctx->h_total;
    // offs[] is int32 and the scan saturates at INT32_MAX instead of wrapping, so
    // an oversized total shows up here; cap the sample table at 2^27 rows.
    if (total < 0 || total > (1 << 27))
        return fail(ctx, BCC_ERR_LIMIT, "too many samples in one call (edges too long or non-finite)");
    const int NS = ops->num_spheres;
    const size_t tiles = ((size_t)std::max(total, 1) + bcc::kMaxTableTile - 1) / bcc::kMaxTableTile;
    BCC_CUDA(ctx, ctx->table.ensure(sizeof(float4) * (size_t)NS * tiles * bcc::kMaxTableTile));
    BCC_CUDA(ctx, ctx->row_edge.ensure(sizeof(int) * (size_t)std::max(total, 1)));
    a.total_rows = total;
    a.table = ctx->table.as<float4>();
    a.row_edge = ctx->row_edge.as<int>();
    a.blobs = ctx->blobs.as<float4>();
    a.env_hdr = ctx->env_hdr.as<float4>();
    a.num_envs = ctx->num_envs;
    a.max_prims = std::max(ctx->max_prims, 1);
    a.blob_smem = ctx->blob_smem;
    a.d_results = d_results;
    // Tile: warps per CTA (tuned, limited by shared memory); edges per CTA.
    int warps = ctx->tune.warps;
    while (warps > 1 && bcc::check_smem_bytes(a.max_prims, G, a.blob_smem, warps) > 200 * 1024) warps >>= 1;
    if (bcc::check_smem_bytes(a.max_prims, G, a.blob_smem, warps) > 220 * 1024)
        return fail(ctx, BCC_ERR_LIMIT, "an environment has too many primitives for shared-memory staging");
    a.warps = warps;
    a.edges_per_cta = clamp_tile(opts && opts->tile_override > 0 ? opts->tile_override : ctx->tune.edges_per_cta, 1,
                                 1 << 20);
    if ((E + a.edges_per_cta - 1) / a.edges_per_cta > 65535)
        a.edges_per_cta = (E + 65534) / 65535;
    a.persistent = ctx->tune.persistent;
    a.queue_min_items = ctx->tune.queue_min_items;
    a.finish_split = ctx->tune.finish_split;
    a.mode = ctx->tune.lanes == 16 ? 5 : 0;  // the plain walk: whole warp or half-warp per pair
    BCC_CUDA(ctx, ctx->work_counter.ensure(64));
    a.work_counter = ctx->work_counter.as<int>();
    return BCC_OK;
}

// Environment codes of the uploaded set (once per upload).
bcc_status ensure_env_code(bcc_ctx* ctx, cudaStream_t st) {
    if (ctx->env_code_ready) return BCC_OK;
    BCC_CUDA(ctx, ctx->env_code.ensure(sizeof(float) * bcc::kEnvCode * (size_t)std::max(ctx->num_envs, 1)));
    BCC_CUDA(ctx, bcc::launch_env_encode(ctx->blobs.as<float4>(), ctx->env_hdr.as<float4>(), ctx->num_envs,
                                         ctx->env_code.as<float>(), st));
    ctx->env_code_ready = true;
    return BCC_OK;
}

// Environment clusters of the inline learned order: k-means (Lloyd, 20
// iterations) over the uploaded set's 32-value codes, K = min(tune.clusters,
// num_envs), seeded deterministically by farthest-point selection from
// environment 0.  The MLP scores each edge's segments once per cluster, with
// the centroid as the environment code.  Recomputed when K changes or the set
// is replaced.  Synchronous (host k-means); called outside any stream capture.
bcc_status ensure_env_clusters(bcc_ctx* ctx, cudaStream_t st) {
    const int N = ctx->num_envs;
    const int K = std::max(1, std::min(ctx->tune.clusters, N));
    if (ctx->cluster_k == K) return BCC_OK;
    bcc_status s = ensure_env_code(ctx, st);
    if (s != BCC_OK) return s;
    constexpr int D = bcc::kEnvCode;
    std::vector<float> code((size_t)N * D);
    BCC_CUDA(ctx, cudaMemcpyAsync(code.data(), ctx->env_code.p, sizeof(float) * code.size(), cudaMemcpyDeviceToHost,
                                  st));
    BCC_CUDA(ctx, cudaStreamSynchronize(st));
    auto d2 = [&](const float* a, const float* b) {
        double t = 0;
        for (int j = 0; j < D; ++j) t += (double)(a[j] - b[j]) * (a[j] - b[j]);
        return t;
    };
    std::vector<float> cen((size_t)K * D);
    std::vector<double> best((size_t)N, 1e300);
    int pick = 0;
    for (int k = 0; k < K; ++k) {
        std::copy(&code[(size_t)pick * D], &code[(size_t)pick * D] + D, &cen[(size_t)k * D]);
        int far = 0;
        for (int i = 0; i < N; ++i) {
            best[i] = std::min(best[i], d2(&code[(size_t)i * D], &cen[(size_t)k * D]));
            if (best[i] > best[far]) far = i;
        }
        pick = far;
    }
    std::vector<int> id((size_t)N, 0);
    for (int it = 0; it < 20; ++it) {
        for (int i = 0; i < N; ++i) {
            double bd = 1e300;
            for (int k = 0; k < K; ++k) {
                const double v = d2(&code[(size_t)i * D], &cen[(size_t)k * D]);
                if (v < bd) {
                    bd = v;
                    id[i] = k;
                }
            }
        }
        std::vector<double> sum((size_t)K * D, 0.0);
        std::vector<int> cnt((size_t)K, 0);
        for (int i = 0; i < N; ++i) {
            cnt[id[i]] += 1;
            for (int j = 0; j < D; ++j) sum[(size_t)id[i] * D + j] += code[(size_t)i * D + j];
        }
        for (int k = 0; k < K; ++k)
            if (cnt[k] > 0)  // an empty cluster keeps its centroid
                for (int j = 0; j < D; ++j) cen[(size_t)k * D + j] = (float)(sum[(size_t)k * D + j] / cnt[k]);
    }
    BCC_CUDA(ctx, ctx->env_cluster.ensure(sizeof(int) * (size_t)std::max(N, 1)));
    BCC_CUDA(ctx, ctx->centroids.ensure(sizeof(float) * cen.size()));
    BCC_CUDA(ctx, cudaMemcpy(ctx->env_cluster.p, id.data(), sizeof(int) * (size_t)N, cudaMemcpyHostToDevice));
    BCC_CUDA(ctx, cudaMemcpy(ctx->centroids.p, cen.data(), sizeof(float) * cen.size(), cudaMemcpyHostToDevice));
    ctx->cluster_k = K;
    return BCC_OK;
}

constexpr int kLearnedRowCap = 16 << 20;  // MLP rows per learned check (1.5 GB of features)

// Learned order: (1) plain probe of each pair's rank 0 (first sample), undecided pairs
// queued with MLP rows for their segments; (2) segment features and tcgen05
// MLP scores; (3) the queued pairs walked in descending segment score.
// Buffers are sized here, outside any stream capture.
bcc_status prepare_learned(bcc_ctx* ctx, bcc::PipelineArgs& a, int row_cap) {
    const long long cap_ll = (long long)a.num_envs * (a.total_rows / bcc::kSegment) + 64;
    const int cap = (int)std::min<long long>(cap_ll, row_cap > 0 ? std::min(row_cap, kLearnedRowCap) : kLearnedRowCap);
    // A queued pair takes at least 4 rows; the probe stops queueing once the
    // rows are spent, so the queue needs cap / 4 entries plus the pairs that
    // were in flight at that moment (the kernel checks the capacity anyway).
    const long long pairs = (long long)a.num_envs * a.num_edges;
    const int q_cap = (int)std::min<long long>(pairs, cap / 4 + (1 << 18));
    BCC_CUDA(ctx, ctx->q_head.ensure(64));
    BCC_CUDA(ctx, ctx->q_pairs.ensure(sizeof(int2) * (size_t)q_cap));
    BCC_CUDA(ctx, ctx->q_rows.ensure(sizeof(int) * (size_t)q_cap));
    BCC_CUDA(ctx, ctx->mlp.x.ensure(sizeof(uint16_t) * bcc::kMlpIn * (size_t)cap));
    BCC_CUDA(ctx, ctx->mlp.logits.ensure(sizeof(float) * (size_t)cap));
    a.q_head = ctx->q_head.as<unsigned long long>();
    a.q_pairs = ctx->q_pairs.as<int2>();
    a.q_rows = ctx->q_rows.as<int>();
    a.q_cap = q_cap;
    a.row_cap = cap;
    a.logits = ctx->mlp.logits.as<float>();
    a.queue_min_items = ctx->tune.queue_min_items;
    a.finish_counter = a.work_counter + 1;
    ctx->learned_rows_dev = reinterpret_cast<int*>(a.q_head);  // the low word counts rows
    ctx->last_learned_inline = false;
    ctx->learned_row_cap = cap;
    ctx->learned_q_cap = q_cap;
    return BCC_OK;
}

bcc_status run_learned(bcc_ctx* ctx, const bcc::RobotOps* ops, bcc::PipelineArgs& a, cudaStream_t st) {
    BCC_CUDA(ctx, cudaMemsetAsync(a.q_head, 0, sizeof(unsigned long long), st));
    cudaEvent_t* ev = a.stage_events;
    BCC_CUDA(ctx, ops->prep(a, st));  // records stage events 1-4
    a.mode = 1;
    BCC_CUDA(ctx, ops->check_mode(a, st));
    // No host round trip: the feature and finish kernels read the queue length
    // and the MLP kernel the row count on the device (capped by the capacities).
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    BCC_CUDA(ctx, ops->queue_features(a, ctx->env_code.as<float>(), ctx->mlp.x.as<uint16_t>(), 16 * std::max(sms, 1),
                                      st));
    BCC_CUDA(ctx, bcc::mlp_forward(ctx->mlp.x.as<uint16_t>(), a.row_cap, ctx->mlp.images.as<uint8_t>(),
                                   ctx->mlp.params.as<float>(), ctx->mlp.logits.as<float>(), a.error_flag,
                                   std::max(sms, 1), st, reinterpret_cast<const int*>(a.q_head)));
    a.mode = 2;
    BCC_CUDA(ctx, ops->check_mode(a, st));
    if (ev) cudaEventRecord(ev[5], st);
    return BCC_OK;
}

// Inline learned order: buffers for K x segments MLP rows and the
// per-(cluster, edge) 32-block permutations, sized outside any stream capture.
bcc_status prepare_inline(bcc_ctx* ctx, bcc::PipelineArgs& a) {
    bcc_status s = ensure_env_clusters(ctx, ctx->stream);
    if (s != BCC_OK) return s;
    const int K = ctx->cluster_k;
    a.total_segs = a.total_rows / bcc::kSegment;
    const size_t rows = (size_t)K * std::max(a.total_segs, 1);
    if (rows > (size_t)kLearnedRowCap * 4)
        return fail(ctx, BCC_ERR_LIMIT, "too many (cluster, segment) rows for the inline learned order");
    BCC_CUDA(ctx, ctx->mlp.x.ensure(sizeof(uint16_t) * bcc::kMlpIn * rows));
    BCC_CUDA(ctx, ctx->mlp.logits.ensure(sizeof(float) * rows));
    BCC_CUDA(ctx, ctx->perms.ensure((size_t)K * std::max(a.num_edges, 1) * bcc::kLanes));
    a.logits = ctx->mlp.logits.as<float>();
    a.env_cluster = ctx->env_cluster.as<int>();
    a.perms = ctx->perms.as<uint8_t>();
    a.row_cap = (int)rows;
    ctx->last_inline_rows = (long long)rows;
    ctx->last_learned_inline = true;
    return BCC_OK;
}

// Inline learned order: FK / self / swept, features of every (cluster,
// segment) row, tcgen05 MLP scores, per-(cluster, edge) permutations, then one
// check in which every pair walks rank 0 (sample 0) and then its other samples
// in its cluster's learned order (mode 4): no queue, no second pass.
// With one cluster the permutation depends on the edge alone, so the FK
// kernel writes each edge's table rows in learned order (lane block pi(t) at
// block position t) and the plain check kernel (mode 0) walks them: the order
// costs the check kernel nothing.  With several clusters the table stays in
// sample order and the check kernel (mode 4) maps ranks through each pair's
// cluster permutation.
bcc_status run_learned_inline(bcc_ctx* ctx, const bcc::RobotOps* ops, bcc::PipelineArgs& a, cudaStream_t st) {
    cudaEvent_t* ev = a.stage_events;
    const int K = ctx->cluster_k;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    BCC_CUDA(ctx, ops->cluster_features(a, ctx->centroids.as<float>(), K, ctx->mlp.x.as<uint16_t>(), st));
    BCC_CUDA(ctx, bcc::mlp_forward(ctx->mlp.x.as<uint16_t>(), a.row_cap, ctx->mlp.images.as<uint8_t>(),
                                   ctx->mlp.params.as<float>(), ctx->mlp.logits.as<float>(), a.error_flag,
                                   std::max(sms, 1), st));
    BCC_CUDA(ctx, ops->cluster_perms(a, K, ctx->perms.as<uint8_t>(), st));
    a.fk_perm = K == 1 ? ctx->perms.as<uint8_t>() : nullptr;
    BCC_CUDA(ctx, ops->prep(a, st));  // records stage events 1-4
    a.mode = K == 1 ? a.mode : 4;  // one cluster: the plain walk (whole or half warp) over the permuted table
    BCC_CUDA(ctx, ops->check_mode(a, st));
    if (ev) cudaEventRecord(ev[5], st);
    return BCC_OK;
}

bcc_status launch_sequence(bcc_ctx* ctx, bcc_robot robot, bcc::PipelineArgs& a, bool learned, cudaStream_t st) {
    const bcc::RobotOps* ops = bcc::robot_ops((int)robot);
    if (!ops) return fail(ctx, BCC_ERR_NOT_SUPPORTED, "robot not built into this library");
    if (learned) return ctx->tune.learned_mode == 0 ? run_learned_inline(ctx, ops, a, st) : run_learned(ctx, ops, a, st);
    BCC_CUDA(ctx, ops->check(a, st));
    return BCC_OK;
}

bool same_tune(const bcc::Tune& x, const bcc::Tune& y) {
    return x.edges_per_cta == y.edges_per_cta && x.warps == y.warps && x.persistent == y.persistent &&
           x.queue_min_items == y.queue_min_items && x.finish_split == y.finish_split &&
           x.learned_mode == y.learned_mode && x.clusters == y.clusters && x.lanes == y.lanes;
}

bcc_status run_check(bcc_ctx* ctx, bcc_robot robot, const float* d_edges, int E, int resolution,
                     uint8_t* d_results, const bcc_opts* opts, cudaStream_t st) {
    bcc::PipelineArgs a;
    bcc_status s = prepare(ctx, robot, d_edges, E, resolution, d_results, opts, st, a);
    if (s != BCC_OK) return s;
    const bool learned = opts && opts->order == BCC_ORDER_LEARNED;
    if (learned) {
        if (!ctx->mlp.ready)
            return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "learned order needs MLP parameters (bcc_mlp_train or bcc_mlp_set_params)");
        s = ensure_env_code(ctx, st);
        if (s != BCC_OK) return s;
        if (opts->learned_row_cap < 0)
            return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "learned_row_cap must be >= 0");
        s = ctx->tune.learned_mode == 0 ? prepare_inline(ctx, a) : prepare_learned(ctx, a, opts->learned_row_cap);
        if (s != BCC_OK) return s;
    }
    const bool graph = opts && opts->use_graph && !ctx->counting && !(opts->tile_override > 0);
    if (!graph) return launch_sequence(ctx, robot, a, learned, st);
    // CUDA graph of everything after the discretisation (whose sample total sizes
    // the launches): replayed while the inputs and configuration are unchanged.
    bcc::GraphCache& G = ctx->graph[learned ? 1 : 0];
    const bool hit = G.exec && G.edges == d_edges && G.results == d_results && G.num_edges == E &&
                     G.resolution == resolution && G.total_rows == a.total_rows && G.robot == (int)robot &&
                     G.row_cap == a.row_cap &&
                     G.env_version == ctx->env_version && same_tune(G.tune, ctx->tune);
    if (!hit) {
        if (G.exec) {
            cudaGraphExecDestroy(G.exec);
            G.exec = nullptr;
        }
        a.stage_events = nullptr;
        cudaGraph_t g = nullptr;
        // Captured on the context's private stream (the caller's may be the legacy
        // default stream, which cannot be captured); launched on the caller's.
        cudaStream_t cs = ctx->capture_stream;
        BCC_CUDA(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        s = launch_sequence(ctx, robot, a, learned, cs);
        cudaError_t ce = cudaStreamEndCapture(cs, &g);
        if (s != BCC_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaStreamEndCapture");
        ce = cudaGraphInstantiate(&G.exec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaGraphInstantiate");
        G.edges = d_edges;
        G.results = d_results;
        G.stream = st;
        G.num_edges = E;
        G.resolution = resolution;
        G.total_rows = a.total_rows;
        G.row_cap = a.row_cap;
        G.robot = (int)robot;
        G.env_version = ctx->env_version;
        G.tune = ctx->tune;
    }
    cudaEvent_t* ev = ctx->profiling ? ctx->ev : nullptr;
    if (ev) cudaEventRecord(ev[1], st);
    BCC_CUDA(ctx, cudaGraphLaunch(G.exec, st));
    if (ev) {
        for (int i = 2; i <= 5; ++i) cudaEventRecord(ev[i], st);
    }
    return BCC_OK;
}

}  // namespace

extern "C" {

bcc_status bcc_create(bcc_ctx** out, int device) {
    if (!out) return BCC_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    bcc_ctx* c = new bcc_ctx();
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->capture_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_total, sizeof(int));
    if (e != cudaSuccess) {
        delete c;
        return BCC_ERR_CUDA;
    }
    *out = c;
    return BCC_OK;
}

void bcc_destroy(bcc_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->h_total) cudaFreeHost(ctx->h_total);
    for (auto& g : ctx->graph)
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->capture_stream) cudaStreamDestroy(ctx->capture_stream);
    delete ctx;
}

const char* bcc_last_error(const bcc_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

bcc_status bcc_set_profiling(bcc_ctx* ctx, int32_t on) {
    if (!ctx) return BCC_ERR_INVALID_ARGUMENT;
    BCC_CUDA(ctx, cudaSetDevice(ctx->device));
    for (auto& e : ctx->ev)
        if (!e) BCC_CUDA(ctx, cudaEventCreate(&e));
    ctx->profiling = on != 0;
    ctx->counting = (on & 2) != 0;
    return BCC_OK;
}

int32_t bcc_work_counters(bcc_ctx* ctx, uint64_t* out, int32_t max_counters) {
    if (!ctx || !out || !ctx->counting || !ctx->counters.p) return -1;
    const int n = std::min<int>(max_counters, bcc::kNumCounters);
    unsigned long long tmp[bcc::kNumCounters];
    if (cudaMemcpy(tmp, ctx->counters.p, sizeof(tmp), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    for (int i = 0; i < n; ++i) out[i] = tmp[i];
    return n;
}

int32_t bcc_stage_times(bcc_ctx* ctx, float* ms, int32_t max_stages) {
    if (!ctx || !ms || !ctx->profiling) return -1;
    int n = std::min(max_stages, 5);
    for (int i = 0; i < n; ++i) {
        if (cudaEventElapsedTime(&ms[i], ctx->ev[i], ctx->ev[i + 1]) != cudaSuccess) return -1;
    }
    return n;
}

int32_t bcc_robot_dof(bcc_robot robot) {
    switch (robot) {
        case BCC_ROBOT_PANDA: return 7;
        case BCC_ROBOT_FETCH: return 8;
        case BCC_ROBOT_BAXTER: return 14;
        default: return -1;
    }
}

int32_t bcc_edge_samples(const float* start, const float* end, int32_t dof, int32_t resolution) {
    if (!start || !end || dof <= 0 || dof > 16) return -1;
    // Host copy of the reference discretisation (src/batch_cc.cu:103-107).
    float ans = 0.0f;
    for (int j = 0; j < dof; ++j) {
        float d = start[j] - end[j];
        ans = std::fmaf(d, d, ans);
    }
    float dist = std::sqrt(ans);
    float nf = std::fmax(std::ceil((dist / 31.0f) * (float)resolution), 1.0f);
    return 32 * (int)nf;
}

}  // extern "C"

namespace {

// Validation + packing shared by bcc_upload_envs and bcc_pack_envs.
bcc_status pack(bcc_ctx* ctx, const bcc_env_soa* envs, std::vector<Rec>& recs, std::vector<int>& off,
                int& max_prims) {
    if (!envs || envs->num_envs < 0) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "null or negative environment set");
    const int N = envs->num_envs;
    const uint32_t* cnt[6] = {envs->num_spheres, envs->num_capsules, envs->num_z_capsules,
                              envs->num_cuboids, envs->num_z_cuboids, envs->num_cylinders};
    const float* rec[6] = {envs->spheres, envs->capsules, envs->z_capsules,
                           envs->cuboids, envs->z_cuboids, envs->cylinders};
    const int width[6] = {4, 8, 8, 15, 15, 8};
    const char* names[6] = {"spheres", "capsules", "z_capsules", "cuboids", "z_cuboids", "cylinders"};
    // ensure_ptr_count_consistent (src/batch_cc.cu:45-56): positive count needs records.
    for (int k = 0; k < 6; ++k) {
        if (!cnt[k]) continue;
        size_t tot = 0;
        for (int i = 0; i < N; ++i) tot += cnt[k][i];
        if (tot > 0 && !rec[k])
            return fail(ctx, BCC_ERR_INVALID_ARGUMENT,
                        std::string("positive ") + names[k] + " count with null records");
    }
    recs.clear();
    off.assign(N + 1, 0);
    size_t pos[6] = {0, 0, 0, 0, 0, 0};
    max_prims = 0;
    for (int i = 0; i < N; ++i) {
        for (int k = 0; k < 5; ++k) {
            uint32_t c = cnt[k] ? cnt[k][i] : 0;
            for (uint32_t j = 0; j < c; ++j) {
                const float* r = rec[k] + (pos[k] + j) * width[k];
                switch (k) {
                    case 0: recs.push_back(rec_sphere(r)); break;
                    case 1: recs.push_back(rec_capsule(r, false)); break;
                    case 2: recs.push_back(rec_capsule(r, true)); break;
                    case 3: recs.push_back(rec_cuboid(r, false)); break;
                    case 4: recs.push_back(rec_cuboid(r, true)); break;
                }
            }
            pos[k] += c;
        }
        if (cnt[5]) pos[5] += cnt[5][i];  // cylinders: never tested (src/utils.cuh:213-245)
        off[i + 1] = (int)recs.size();
        max_prims = std::max(max_prims, off[i + 1] - off[i]);
        if (recs.size() > (size_t)0x7fffffff) return fail(ctx, BCC_ERR_LIMIT, "too many primitives");
    }
    if (max_prims > 4095) return fail(ctx, BCC_ERR_LIMIT, "more than 4095 primitives in one environment");
    return BCC_OK;
}

// Device arena: per environment a blob of its rounded-box records followed by
// its interval-mask cull tables, and a 2 x float4 header.  The check kernel
// stages the records into shared memory and reads the mask tables through L1.
struct Arena {
    std::vector<float> blob;     // concatenated blobs (float words, 16-byte granules)
    std::vector<float> hdr;      // [N][8]
    size_t max_record_bytes = 0;
    // Cull grid shared by every environment of the set: slab s of axis a is
    // [bnd[a][s], bnd[a][s + 1]).
    float bnd[3][bcc::kGridSlabs + 1] = {};
};

// Largest slab s in [0, K) with bnd[s] <= x (0 below the first boundary);
// the device lookup (swept_kernel) compares against the same floats.
int slab_of(const float* bnd, double x) {
    int s = 0;
    for (int i = 1; i < bcc::kGridSlabs; ++i)
        if ((double)bnd[i] <= x) s = i;
    return s;
}

// One cull grid serves all environments of the set, so an edge's slab ranges
// depend on the edge alone and are found once per edge (swept_kernel).  The
// kGridSlabs slabs of an axis run from below every primitive AABB to above
// them, split at quantiles of the primitives' centres: slabs are narrow where
// primitives are dense.
void build_arena(const std::vector<Rec>& recs, const std::vector<int>& off, Arena& A) {
    const int N = (int)off.size() - 1;
    constexpr int K = bcc::kGridSlabs;
    constexpr int TRI = bcc::kGridTri;
    A.blob.clear();
    A.hdr.assign((size_t)N * 8, 0.0f);
    for (int a = 0; a < 3; ++a) {
        std::vector<double> c;
        double lo = 1e30, hi = -1e30;
        c.reserve(recs.size());
        for (const Rec& r : recs) {
            c.push_back(r.v[a]);
            lo = std::min(lo, (double)r.v[a] - r.v[16 + a]);
            hi = std::max(hi, (double)r.v[a] + r.v[16 + a]);
        }
        float* b = A.bnd[a];
        if (c.empty()) {
            for (int i = 0; i <= K; ++i) b[i] = (float)i;
            continue;
        }
        std::sort(c.begin(), c.end());
        b[0] = std::nextafter((float)(lo - 1e-4), -INFINITY);
        b[K] = std::nextafter((float)(hi + 1e-4), INFINITY);
        for (int i = 1; i < K; ++i) {
            const double q = c[std::min(c.size() - 1, (size_t)((double)i * c.size() / K))];
            b[i] = std::min(std::max((float)q, std::nextafter(b[i - 1], INFINITY)), b[K]);
        }
        for (int i = K - 1; i >= 1; --i)  // strictly increasing up to b[K]
            if (b[i] >= b[i + 1]) b[i] = std::nextafter(b[i + 1], -INFINITY);
    }
    for (int i = 0; i < N; ++i) {
        const int p0 = off[i], np = off[i + 1] - off[i];
        const int W = np > 0 ? (np + 63) / 64 : 0;
        const size_t start = A.blob.size();  // in floats, multiple of 4
        for (int p = 0; p < np; ++p) {
            const Rec& r = recs[p0 + p];
            for (int k = 0; k < 20; ++k) A.blob.push_back(r.v[k]);
        }
        if (np > 0) {
            // Slab range of each primitive's AABB, widened by 1e-5 m so that the
            // FP32 swept boxes on the device can only over-include.
            std::vector<int> s0(3 * (size_t)np), s1(3 * (size_t)np);
            for (int p = 0; p < np; ++p) {
                const Rec& r = recs[p0 + p];
                for (int a = 0; a < 3; ++a) {
                    s0[3 * p + a] = slab_of(A.bnd[a], (double)r.v[a] - r.v[16 + a] - 1e-5);
                    s1[3 * p + a] = slab_of(A.bnd[a], (double)r.v[a] + r.v[16 + a] + 1e-5);
                }
            }
            std::vector<uint64_t> m((size_t)3 * TRI * W, 0);
            for (int a = 0; a < 3; ++a)
                for (int i0 = 0; i0 < K; ++i0)
                    for (int i1 = i0; i1 < K; ++i1) {
                        uint64_t* dst = &m[((size_t)a * TRI + bcc::tri_index(i0, i1)) * W];
                        for (int p = 0; p < np; ++p)
                            if (s0[3 * p + a] <= i1 && s1[3 * p + a] >= i0) dst[p >> 6] |= 1ull << (p & 63);
                    }
            const size_t words = m.size() * 2;
            const size_t at = A.blob.size();
            A.blob.resize(at + words);
            std::memcpy(&A.blob[at], m.data(), m.size() * sizeof(uint64_t));
        }
        A.max_record_bytes = std::max(A.max_record_bytes, (size_t)np * sizeof(Rec));
        const uint32_t off16 = (uint32_t)(start / 4);  // float4 units
        const uint32_t shape = (uint32_t)np | ((uint32_t)W << 16);
        float* h = &A.hdr[(size_t)i * 8];
        std::memcpy(&h[3], &off16, 4);
        std::memcpy(&h[7], &shape, 4);
    }
    if (A.blob.empty()) A.blob.assign(4, 0.0f);
}

}  // namespace

extern "C" {

bcc_status bcc_pack_envs(const bcc_env_soa* envs, float* records, int32_t* env_offsets, int64_t* num_records,
                         int32_t* max_prims_per_env) {
    std::vector<Rec> recs;
    std::vector<int> off;
    int max_prims = 0;
    bcc_status s = pack(nullptr, envs, recs, off, max_prims);
    if (s != BCC_OK) return s;
    if (num_records) *num_records = (int64_t)recs.size();
    if (max_prims_per_env) *max_prims_per_env = max_prims;
    if (records && !recs.empty()) std::memcpy(records, recs.data(), recs.size() * sizeof(Rec));
    if (env_offsets) std::memcpy(env_offsets, off.data(), off.size() * sizeof(int));
    return BCC_OK;
}

bcc_status bcc_upload_envs(bcc_ctx* ctx, const bcc_env_soa* envs) {
    if (!ctx) return BCC_ERR_INVALID_ARGUMENT;
    std::vector<Rec> recs;
    std::vector<int> off;
    int max_prims = 0;
    bcc_status s = pack(ctx, envs, recs, off, max_prims);
    if (s != BCC_OK) return s;
    const int N = envs->num_envs;
    Arena A;
    build_arena(recs, off, A);
    const size_t blob_smem = (A.max_record_bytes + 15) & ~(size_t)15;
    if (blob_smem > 160 * 1024)
        return fail(ctx, BCC_ERR_LIMIT, "an environment's primitives do not fit shared-memory staging (max 2048)");
    if (A.blob.size() / 4 > 0xffffffffull) return fail(ctx, BCC_ERR_LIMIT, "environment arena too large");
    BCC_CUDA(ctx, cudaSetDevice(ctx->device));
    BCC_CUDA(ctx, ctx->blobs.ensure(A.blob.size() * sizeof(float)));
    BCC_CUDA(ctx, ctx->env_hdr.ensure(std::max<size_t>(1, A.hdr.size()) * sizeof(float)));
    BCC_CUDA(ctx, cudaMemcpy(ctx->blobs.p, A.blob.data(), A.blob.size() * sizeof(float), cudaMemcpyHostToDevice));
    if (N > 0)
        BCC_CUDA(ctx, cudaMemcpy(ctx->env_hdr.p, A.hdr.data(), A.hdr.size() * sizeof(float), cudaMemcpyHostToDevice));
    ctx->num_envs = N;
    ctx->max_prims = max_prims;
    ctx->blob_smem = blob_smem;
    BCC_CUDA(ctx, ctx->grid_bounds.ensure(sizeof(A.bnd)));
    BCC_CUDA(ctx, cudaMemcpy(ctx->grid_bounds.p, A.bnd, sizeof(A.bnd), cudaMemcpyHostToDevice));
    ctx->env_code_ready = false;
    ctx->cluster_k = 0;
    ctx->env_version += 1;
    return BCC_OK;
}

bcc_status bcc_check_device(bcc_ctx* ctx, bcc_robot robot, const float* d_edges, int32_t num_edges,
                            int32_t resolution, uint8_t* d_results, const bcc_opts* opts, void* stream) {
    if (!ctx) return BCC_ERR_INVALID_ARGUMENT;
    if (ctx->num_envs < 0) return fail(ctx, BCC_ERR_NO_ENVS, "no environments uploaded");
    if (num_edges < 0 || resolution <= 0) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "bad edge count or resolution");
    if (num_edges == 0 || ctx->num_envs == 0) return BCC_OK;
    if (!d_edges || !d_results) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "null edges or results");
    BCC_CUDA(ctx, cudaSetDevice(ctx->device));
    return run_check(ctx, robot, d_edges, num_edges, resolution, d_results, opts,
                     static_cast<cudaStream_t>(stream));
}

bcc_status bcc_check(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges, int32_t resolution,
                     uint8_t* results, const bcc_opts* opts) {
    if (!ctx) return BCC_ERR_INVALID_ARGUMENT;
    if (ctx->num_envs < 0) return fail(ctx, BCC_ERR_NO_ENVS, "no environments uploaded");
    if (num_edges < 0 || resolution <= 0) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "bad edge count or resolution");
    const int dof = bcc_robot_dof(robot);
    if (dof < 0) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "unknown robot");
    if (num_edges == 0 || ctx->num_envs == 0) return BCC_OK;
    if (!edges || !results) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "null edges or results");
    BCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t eb = sizeof(float) * 2 * (size_t)dof * num_edges;
    const size_t rb = (size_t)num_edges * ctx->num_envs;
    BCC_CUDA(ctx, ctx->edges.ensure(eb));
    BCC_CUDA(ctx, ctx->results.ensure(rb));
    cudaStream_t st = ctx->stream;
    BCC_CUDA(ctx, cudaMemcpyAsync(ctx->edges.p, edges, eb, cudaMemcpyHostToDevice, st));
    bcc_status s = run_check(ctx, robot, ctx->edges.as<float>(), num_edges, resolution,
                             ctx->results.as<uint8_t>(), opts, st);
    if (s != BCC_OK) return s;
    BCC_CUDA(ctx, cudaMemcpyAsync(results, ctx->results.p, rb, cudaMemcpyDeviceToHost, st));
    BCC_CUDA(ctx, cudaStreamSynchronize(st));
    int flag = 0;
    BCC_CUDA(ctx, cudaMemcpy(&flag, ctx->error_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag & 4) return fail(ctx, BCC_ERR_TIMEOUT, "a walk exceeded its step bound");
    if (flag) return fail(ctx, BCC_ERR_TIMEOUT, "a bounded device wait gave up (bulk copy did not complete)");
    return BCC_OK;
}

// Train the collision-likelihood MLP on checker-labelled samples drawn from
// the uploaded environments and the given (host) edges.
bcc_status bcc_mlp_train(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges, int32_t resolution,
                         int64_t num_samples, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                         float* h_epoch_loss, float* h_positive_fraction) {
    if (!ctx) return BCC_ERR_INVALID_ARGUMENT;
    if (ctx->num_envs <= 0) return fail(ctx, BCC_ERR_NO_ENVS, "no environments uploaded");
    if (!edges || num_edges <= 0 || num_samples <= 0 || epochs <= 0 || batch < 128 || resolution <= 0)
        return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "bad training arguments");
    if (!ctx->mlp.ready) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "set initial MLP parameters first");
    BCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int dof = bcc_robot_dof(robot);
    if (dof < 0) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "unknown robot");
    cudaStream_t st = ctx->stream;
    BCC_CUDA(ctx, ctx->edges.ensure(sizeof(float) * 2 * (size_t)dof * num_edges));
    BCC_CUDA(ctx, cudaMemcpy(ctx->edges.p, edges, sizeof(float) * 2 * (size_t)dof * num_edges, cudaMemcpyHostToDevice));
    bcc::PipelineArgs a;
    bcc_status s = prepare(ctx, robot, ctx->edges.as<float>(), num_edges, resolution, nullptr, nullptr, st, a);
    if (s != BCC_OK) return s;
    BCC_CUDA(ctx, bcc::robot_ops((int)robot)->prep(a, st));
    s = ensure_env_code(ctx, st);
    if (s != BCC_OK) return s;
    bcc::MlpState& m = ctx->mlp;
    BCC_CUDA(ctx, m.x.ensure(sizeof(uint16_t) * bcc::kMlpIn * (size_t)num_samples));
    BCC_CUDA(ctx, m.y.ensure((size_t)num_samples));
    BCC_CUDA(ctx, bcc::robot_ops((int)robot)->training_rows(a, ctx->env_code.as<float>(), num_samples, seed,
                                            m.x.as<uint16_t>(), m.y.as<uint8_t>(), st));
    BCC_CUDA(ctx, cudaStreamSynchronize(st));
    if (h_positive_fraction) {
        std::vector<uint8_t> yy((size_t)num_samples);
        BCC_CUDA(ctx, cudaMemcpy(yy.data(), m.y.p, yy.size(), cudaMemcpyDeviceToHost));
        size_t pos = 0;
        for (uint8_t v : yy) pos += v;
        *h_positive_fraction = (float)pos / (float)yy.size();
    }
    const long long nb = num_samples / batch;
    for (int ep = 0; ep < epochs; ++ep) {
        double tot = 0.0;
        for (long long b = 0; b < nb; ++b) {
            float loss = 0.0f;
            s = bcc_mlp_train_step(ctx, m.x.as<uint16_t>() + (size_t)b * batch * bcc::kMlpIn, m.y.as<uint8_t>() + (size_t)b * batch,
                                   batch, lr, &loss);
            if (s != BCC_OK) return s;
            tot += loss;
        }
        if (h_epoch_loss) h_epoch_loss[ep] = (float)(tot / (double)(nb * batch));
    }
    return BCC_OK;
}

// Held-out evaluation on fresh samples: metrics[0] mean BCE, [1] misprediction
// rate (sign of the logit vs the checker's label), [2] false-positive rate,
// [3] false-negative rate, [4] positive fraction.
bcc_status bcc_mlp_evaluate(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges, int32_t resolution,
                            int64_t num_samples, uint64_t seed, float* h_metrics) {
    if (!ctx || !h_metrics) return BCC_ERR_INVALID_ARGUMENT;
    if (ctx->num_envs <= 0) return fail(ctx, BCC_ERR_NO_ENVS, "no environments uploaded");
    if (!ctx->mlp.ready || !edges || num_edges <= 0 || num_samples <= 0) return BCC_ERR_INVALID_ARGUMENT;
    BCC_CUDA(ctx, cudaSetDevice(ctx->device));
    const int dof = bcc_robot_dof(robot);
    cudaStream_t st = ctx->stream;
    BCC_CUDA(ctx, ctx->edges.ensure(sizeof(float) * 2 * (size_t)dof * num_edges));
    BCC_CUDA(ctx, cudaMemcpy(ctx->edges.p, edges, sizeof(float) * 2 * (size_t)dof * num_edges, cudaMemcpyHostToDevice));
    bcc::PipelineArgs a;
    bcc_status s = prepare(ctx, robot, ctx->edges.as<float>(), num_edges, resolution, nullptr, nullptr, st, a);
    if (s != BCC_OK) return s;
    BCC_CUDA(ctx, bcc::robot_ops((int)robot)->prep(a, st));
    s = ensure_env_code(ctx, st);
    if (s != BCC_OK) return s;
    bcc::MlpState& m = ctx->mlp;
    BCC_CUDA(ctx, m.x.ensure(sizeof(uint16_t) * bcc::kMlpIn * (size_t)num_samples));
    BCC_CUDA(ctx, m.y.ensure((size_t)num_samples));
    BCC_CUDA(ctx, m.logits.ensure(sizeof(float) * (size_t)num_samples));
    BCC_CUDA(ctx, bcc::robot_ops((int)robot)->training_rows(a, ctx->env_code.as<float>(), num_samples, seed,
                                            m.x.as<uint16_t>(), m.y.as<uint8_t>(), st));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    BCC_CUDA(ctx, cudaMemsetAsync(a.error_flag, 0, sizeof(int), st));
    BCC_CUDA(ctx, bcc::mlp_forward(m.x.as<uint16_t>(), (int)num_samples, m.images.as<uint8_t>(), m.params.as<float>(),
                                   m.logits.as<float>(), a.error_flag, std::max(sms, 1), st));
    BCC_CUDA(ctx, cudaStreamSynchronize(st));
    std::vector<uint8_t> yy((size_t)num_samples);
    std::vector<float> zz((size_t)num_samples);
    BCC_CUDA(ctx, cudaMemcpy(yy.data(), m.y.p, yy.size(), cudaMemcpyDeviceToHost));
    BCC_CUDA(ctx, cudaMemcpy(zz.data(), m.logits.p, zz.size() * sizeof(float), cudaMemcpyDeviceToHost));
    double loss = 0;
    long long wrong = 0, fp = 0, fn = 0, pos = 0;
    for (size_t i = 0; i < yy.size(); ++i) {
        const double z = zz[i], y = yy[i];
        loss += std::max(z, 0.0) - z * y + std::log1p(std::exp(-std::fabs(z)));
        const bool pred = z > 0;
        pos += yy[i];
        if (pred != (yy[i] != 0)) {
            ++wrong;
            if (pred) ++fp; else ++fn;
        }
    }
    const double n = (double)yy.size();
    h_metrics[0] = (float)(loss / n);
    h_metrics[1] = (float)(wrong / n);
    h_metrics[2] = (float)(fp / n);
    h_metrics[3] = (float)(fn / n);
    h_metrics[4] = (float)(pos / n);
    return BCC_OK;
}

}  // extern "C"

namespace {

// The learned order's population over the uploaded environments and the given
// host edges: the probe (plain walk of every pair's rank 0, queue threshold
// min_items) queues the pairs still undecided with at least min_items items
// left; each segment of a queued pair gets its MLP feature row (mlp.x, at its
// scored sample), each sample its environment verdict (mlp.lab, 8 per row) and
// each scored sample its label (mlp.y; rows the row budget left unfilled keep
// the label 0xff).  R = rows handed out.
bcc_status queue_population(bcc_ctx* ctx, bcc_robot robot, const float* edges, int E, int resolution, int min_items,
                            bcc::PipelineArgs& a, int& R) {
    const int dof = bcc_robot_dof(robot);
    const bcc::RobotOps* ops = bcc::robot_ops((int)robot);
    if (dof < 0 || !ops) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "unknown robot");
    if (!edges || E <= 0 || resolution <= 0 || min_items < 0)
        return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "bad edges, resolution or queue threshold");
    BCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t eb = sizeof(float) * 2 * (size_t)dof * E;
    BCC_CUDA(ctx, ctx->edges.ensure(eb));
    BCC_CUDA(ctx, cudaMemcpy(ctx->edges.p, edges, eb, cudaMemcpyHostToDevice));
    BCC_CUDA(ctx, ctx->results.ensure((size_t)E * ctx->num_envs));
    bcc_status s = prepare(ctx, robot, ctx->edges.as<float>(), E, resolution, ctx->results.as<uint8_t>(), nullptr, st, a);
    if (s != BCC_OK) return s;
    if ((s = ensure_env_code(ctx, st)) != BCC_OK) return s;
    if ((s = prepare_learned(ctx, a, 0)) != BCC_OK) return s;
    bcc::MlpState& m = ctx->mlp;
    BCC_CUDA(ctx, m.lab.ensure((size_t)a.row_cap * bcc::kSegment));
    BCC_CUDA(ctx, m.y.ensure((size_t)a.row_cap));
    BCC_CUDA(ctx, cudaMemsetAsync(m.y.p, 0xff, (size_t)a.row_cap, st));
    a.queue_min_items = min_items;
    BCC_CUDA(ctx, cudaMemsetAsync(a.q_head, 0, sizeof(unsigned long long), st));
    BCC_CUDA(ctx, ops->prep(a, st));
    a.mode = 1;
    BCC_CUDA(ctx, ops->check_mode(a, st));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    BCC_CUDA(ctx, ops->queue_features(a, ctx->env_code.as<float>(), m.x.as<uint16_t>(), 16 * std::max(sms, 1), st));
    BCC_CUDA(ctx, ops->queue_labels(a, m.lab.as<uint8_t>(), m.y.as<uint8_t>(), 16 * std::max(sms, 1), st));
    unsigned long long head = 0;
    BCC_CUDA(ctx, cudaMemcpyAsync(&head, a.q_head, sizeof(head), cudaMemcpyDeviceToHost, st));
    BCC_CUDA(ctx, cudaStreamSynchronize(st));
    R = (int)std::min<long long>((long long)(uint32_t)head, a.row_cap);
    return BCC_OK;
}

}  // namespace

extern "C" {

bcc_status bcc_mlp_train_queued(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges,
                                int32_t resolution, int32_t queue_min_items, int64_t num_samples, int32_t epochs,
                                int32_t batch, float lr, uint64_t seed, float* h_epoch_loss,
                                float* h_positive_fraction, int64_t* h_rows) {
    if (!ctx) return BCC_ERR_INVALID_ARGUMENT;
    if (ctx->num_envs <= 0) return fail(ctx, BCC_ERR_NO_ENVS, "no environments uploaded");
    if (num_samples <= 0 || epochs <= 0 || batch < 128)
        return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "bad training arguments");
    if (!ctx->mlp.ready) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "set initial MLP parameters first");
    bcc::PipelineArgs a;
    int R = 0;
    bcc_status s = queue_population(ctx, robot, edges, num_edges, resolution, queue_min_items, a, R);
    if (s != BCC_OK) return s;
    bcc::MlpState& m = ctx->mlp;
    // Seeded shuffle of the filled rows (label 0 or 1), at most num_samples of them.
    std::vector<uint8_t> yy((size_t)R);
    if (R > 0) BCC_CUDA(ctx, cudaMemcpy(yy.data(), m.y.p, yy.size(), cudaMemcpyDeviceToHost));
    std::vector<int> idx;
    idx.reserve(yy.size());
    for (int i = 0; i < R; ++i)
        if (yy[i] <= 1) idx.push_back(i);
    std::mt19937_64 rng(seed);
    std::shuffle(idx.begin(), idx.end(), rng);
    if ((int64_t)idx.size() > num_samples) idx.resize((size_t)num_samples);
    const int used = (int)idx.size();
    if (h_rows) *h_rows = used;
    if (used < batch) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "the queued population has fewer rows than one batch");
    size_t pos = 0;
    for (int i : idx) pos += yy[i];
    if (h_positive_fraction) *h_positive_fraction = (float)((double)pos / used);
    BCC_CUDA(ctx, m.perm.ensure(sizeof(int) * (size_t)used));
    BCC_CUDA(ctx, m.x2.ensure(sizeof(uint16_t) * bcc::kMlpIn * (size_t)used));
    BCC_CUDA(ctx, m.y2.ensure((size_t)used));
    BCC_CUDA(ctx, cudaMemcpy(m.perm.p, idx.data(), sizeof(int) * (size_t)used, cudaMemcpyHostToDevice));
    BCC_CUDA(ctx, bcc::launch_gather_rows(m.x.as<uint16_t>(), m.y.as<uint8_t>(), m.perm.as<int>(), used,
                                          m.x2.as<uint16_t>(), m.y2.as<uint8_t>(), ctx->stream));
    const long long nb = used / batch;
    for (int ep = 0; ep < epochs; ++ep) {
        double tot = 0.0;
        for (long long b = 0; b < nb; ++b) {
            float loss = 0.0f;
            s = bcc_mlp_train_step(ctx, m.x2.as<uint16_t>() + (size_t)b * batch * bcc::kMlpIn,
                                   m.y2.as<uint8_t>() + (size_t)b * batch, batch, lr, &loss);
            if (s != BCC_OK) return s;
            tot += loss;
        }
        if (h_epoch_loss) h_epoch_loss[ep] = (float)(tot / (double)(nb * batch));
    }
    return BCC_OK;
}

bcc_status bcc_mlp_rank_metrics(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges,
                                int32_t resolution, int32_t queue_min_items, double* h_metrics,
                                int32_t max_metrics) {
    if (!ctx || !h_metrics || max_metrics < 0) return BCC_ERR_INVALID_ARGUMENT;
    if (ctx->num_envs <= 0) return fail(ctx, BCC_ERR_NO_ENVS, "no environments uploaded");
    if (!ctx->mlp.ready) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "learned order needs MLP parameters");
    bcc::PipelineArgs a;
    int R = 0;
    bcc_status s = queue_population(ctx, robot, edges, num_edges, resolution, queue_min_items, a, R);
    if (s != BCC_OK) return s;
    bcc::MlpState& m = ctx->mlp;
    cudaStream_t st = ctx->stream;
    BCC_CUDA(ctx, m.logits.ensure(sizeof(float) * (size_t)std::max(R, 1)));
    s = bcc_mlp_forward(ctx, m.x.p, R, m.logits.as<float>(), st);
    if (s != BCC_OK) return s;
    BCC_CUDA(ctx, cudaStreamSynchronize(st));
    unsigned long long head = 0;
    BCC_CUDA(ctx, cudaMemcpy(&head, a.q_head, sizeof(head), cudaMemcpyDeviceToHost));
    const int entries = (int)std::min<long long>((long long)(head >> 32), a.q_cap);
    std::vector<int2> qp((size_t)entries);
    std::vector<int> qr((size_t)entries), steps((size_t)num_edges);
    std::vector<float> z((size_t)R);
    std::vector<uint8_t> lab((size_t)R * bcc::kSegment);
    if (entries > 0) {
        BCC_CUDA(ctx, cudaMemcpy(qp.data(), a.q_pairs, sizeof(int2) * qp.size(), cudaMemcpyDeviceToHost));
        BCC_CUDA(ctx, cudaMemcpy(qr.data(), a.q_rows, sizeof(int) * qr.size(), cudaMemcpyDeviceToHost));
    }
    BCC_CUDA(ctx, cudaMemcpy(steps.data(), a.steps, sizeof(int) * steps.size(), cudaMemcpyDeviceToHost));
    if (R > 0) {
        BCC_CUDA(ctx, cudaMemcpy(z.data(), m.logits.p, sizeof(float) * z.size(), cudaMemcpyDeviceToHost));
        BCC_CUDA(ctx, cudaMemcpy(lab.data(), m.lab.p, lab.size(), cudaMemcpyDeviceToHost));
    }
    // Per queued pair: sample ranks the walk after the probe takes until its
    // first hit (all of them for a collision-free pair) in the plain order
    // (reference ranks 1, 2, ...), the learned order (segments by descending
    // score, ties by index, each from its last sample; the probed sample 0 is
    // walked again) and a perfect order (the first colliding sample first).
    double pairs = 0, coll = 0, rows = 0, pos = 0, wrong = 0;
    double w_plain = 0, w_learn = 0, w_perf = 0, c_plain = 0, c_learn = 0, c_perf = 0;
    std::vector<std::pair<float, uint8_t>> scored;
    scored.reserve((size_t)R);
    for (int i = 0; i < entries; ++i) {
        const int ro = qr[i];
        if (ro < 0) continue;
        const int n = steps[qp[i].x];
        const int S = bcc::kLanes * n, nseg = S / bcc::kSegment;
        if (ro + nseg > R) continue;
        const uint8_t* L = lab.data() + (size_t)ro * bcc::kSegment;
        pairs += 1;
        for (int j = 0; j < nseg; ++j) {
            const uint8_t yj = L[j * bcc::kSegment + bcc::kSegment - 1];
            scored.emplace_back(z[ro + j], yj);
            rows += 1;
            pos += yj;
            wrong += ((z[ro + j] > 0.0f) != (yj != 0)) ? 1 : 0;
        }
        int r_plain = -1;  // reference rank r -> sample (r % 32) * n + r / 32
        for (int r = 1; r < S && r_plain < 0; ++r)
            if (L[(r & 31) * n + (r >> 5)]) r_plain = r;
        std::vector<int> order((size_t)nseg);
        for (int j = 0; j < nseg; ++j) order[j] = j;
        std::stable_sort(order.begin(), order.end(), [&](int u, int v) {
            const float zu = std::isnan(z[ro + u]) ? -INFINITY : z[ro + u];
            const float zv = std::isnan(z[ro + v]) ? -INFINITY : z[ro + v];
            return zu > zv;
        });
        int r_learn = -1;
        for (int p = 0; p < S && r_learn < 0; ++p) {
            const int k = order[p / bcc::kSegment] * bcc::kSegment + (bcc::kSegment - 1 - p % bcc::kSegment);
            if (L[k]) r_learn = p + 1;
        }
        if (r_plain > 0) {
            coll += 1;
            c_plain += r_plain;
            c_learn += r_learn;
            c_perf += 1;
            w_plain += r_plain;
            w_learn += r_learn;
            w_perf += 1;
        } else {
            w_plain += S - 1;
            w_learn += S;
            w_perf += S - 1;
        }
    }
    // AUC of the segment scores against the scored samples' labels (ties half).
    std::sort(scored.begin(), scored.end(), [](const auto& u, const auto& v) { return u.first < v.first; });
    double rank_sum = 0, npos = 0;
    for (size_t i = 0; i < scored.size();) {
        size_t j = i;
        while (j < scored.size() && scored[j].first == scored[i].first) ++j;
        const double avg = 0.5 * (double)(i + 1 + j);
        for (size_t k = i; k < j; ++k)
            if (scored[k].second) {
                rank_sum += avg;
                npos += 1;
            }
        i = j;
    }
    const double nneg = (double)scored.size() - npos;
    const double auc = npos > 0 && nneg > 0 ? (rank_sum - npos * (npos + 1) / 2) / (npos * nneg) : NAN;
    const double cp = std::max(coll, 1.0), qp_n = std::max(pairs, 1.0);
    const double metrics[13] = {pairs, rows, coll / qp_n, rows > 0 ? pos / rows : NAN, auc,
                                c_plain / cp, c_learn / cp, c_perf / cp,
                                w_plain / qp_n, w_learn / qp_n, w_perf / qp_n,
                                c_plain > c_perf ? (c_plain - c_learn) / (c_plain - c_perf) : NAN,
                                rows > 0 ? wrong / rows : NAN};
    for (int i = 0; i < std::min<int>(max_metrics, 13); ++i) h_metrics[i] = metrics[i];
    return BCC_OK;
}

bcc_status bcc_env_code(bcc_ctx* ctx, float* h_code, int32_t num_envs) {
    if (!ctx || !h_code) return BCC_ERR_INVALID_ARGUMENT;
    if (ctx->num_envs < 0) return fail(ctx, BCC_ERR_NO_ENVS, "no environments uploaded");
    if (num_envs != ctx->num_envs) return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "num_envs differs from the uploaded set");
    if (num_envs == 0) return BCC_OK;
    BCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    bcc_status s = ensure_env_code(ctx, st);
    if (s != BCC_OK) return s;
    BCC_CUDA(ctx, cudaMemcpyAsync(h_code, ctx->env_code.p, sizeof(float) * bcc::kEnvCode * (size_t)num_envs,
                                  cudaMemcpyDeviceToHost, st));
    BCC_CUDA(ctx, cudaStreamSynchronize(st));
    return BCC_OK;
}

int64_t bcc_last_learned_rows(const bcc_ctx* ctx) {
    if (ctx && ctx->last_learned_inline) return ctx->last_inline_rows;
    if (!ctx || !ctx->learned_rows_dev) return -1;
    int rows = 0;
    if (cudaMemcpy(&rows, ctx->learned_rows_dev, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return std::min(rows, ctx->learned_row_cap);
}

int64_t bcc_last_learned_pairs(const bcc_ctx* ctx) {
    if (ctx && ctx->last_learned_inline) return 0;  // the inline order queues nothing
    if (!ctx || !ctx->learned_rows_dev) return -1;
    unsigned long long head = 0;  // entries << 32 | rows
    if (cudaMemcpy(&head, ctx->learned_rows_dev, sizeof(head), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return std::min<int64_t>((int64_t)(head >> 32), ctx->learned_q_cap);
}

// Launch configuration (BCC_LAUNCH_CONFIG_LEN values): [0] edges per CTA,
// [1] warps per CTA, [2] persistent kernel (0/1), [3] learned-order queue
// threshold (items), [4] learned-order finish: 1 = each queued pair split over
// a CTA's warps, 0 = one warp per pair, [5] learned order: 0 = inline, 1 =
// queued, [6] inline learned order: environment clusters (1..64), [7] lanes
// per walking pair in the plain-order walk (32, or 16: half-warps).
bcc_status bcc_get_launch_config(const bcc_ctx* ctx, int32_t* cfg) {
    if (!ctx || !cfg) return BCC_ERR_INVALID_ARGUMENT;
    cfg[0] = ctx->tune.edges_per_cta;
    cfg[1] = ctx->tune.warps;
    cfg[2] = ctx->tune.persistent;
    cfg[3] = ctx->tune.queue_min_items;
    cfg[4] = ctx->tune.finish_split;
    cfg[5] = ctx->tune.learned_mode;
    cfg[6] = ctx->tune.clusters;
    cfg[7] = ctx->tune.lanes;
    return BCC_OK;
}

bcc_status bcc_set_launch_config(bcc_ctx* ctx, const int32_t* cfg) {
    if (!ctx || !cfg) return BCC_ERR_INVALID_ARGUMENT;
    if (cfg[0] < 1 || cfg[0] > 4096 || (cfg[1] != 1 && cfg[1] != 2 && cfg[1] != 4 && cfg[1] != 8) ||
        (cfg[2] != 0 && cfg[2] != 1) || cfg[3] < 0 || (cfg[4] != 0 && cfg[4] != 1) ||
        (cfg[5] != 0 && cfg[5] != 1) || cfg[6] < 1 || cfg[6] > 64 || (cfg[7] != 32 && cfg[7] != 16))
        return fail(ctx, BCC_ERR_INVALID_ARGUMENT, "bad launch configuration");
    ctx->tune.edges_per_cta = cfg[0];
    ctx->tune.warps = cfg[1];
    ctx->tune.persistent = cfg[2];
    ctx->tune.queue_min_items = cfg[3];
    ctx->tune.finish_split = cfg[4];
    ctx->tune.learned_mode = cfg[5];
    ctx->tune.clusters = cfg[6];
    ctx->tune.lanes = cfg[7];
    return BCC_OK;
}

// Time each candidate configuration on the given edges against the uploaded
// environments (1 capturing check + the median of 5 timed graph replays, CUDA
// events, L2 overwritten before each) and keep the fastest.
bcc_status bcc_autotune(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges, int32_t resolution,
                        int32_t order, int32_t* chosen) {
    if (!ctx) return BCC_ERR_INVALID_ARGUMENT;
    if (ctx->num_envs <= 0) return fail(ctx, BCC_ERR_NO_ENVS, "no environments uploaded");
    const int dof = bcc_robot_dof(robot);
    if (!edges || num_edges <= 0 || dof < 0 || resolution <= 0) return BCC_ERR_INVALID_ARGUMENT;
    BCC_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t eb = sizeof(float) * 2 * (size_t)dof * num_edges;
    BCC_CUDA(ctx, ctx->edges.ensure(eb));
    BCC_CUDA(ctx, ctx->results.ensure((size_t)num_edges * ctx->num_envs));
    BCC_CUDA(ctx, cudaMemcpy(ctx->edges.p, edges, eb, cudaMemcpyHostToDevice));
    // One full check captures the configuration's graph (everything after the
    // discretisation, which depends only on the edges); then the median of
    // kTuneReps timed replays of that graph, each after L2 was overwritten
    // (untimed) so that no replay starts on the previous one's cached tables.
    // Timing the replays alone keeps the host's per-check work (the sample
    // count read back) out of the comparison.
    constexpr int kTuneReps = 5;
    constexpr size_t kFlushBytes = 256u << 20;  // twice the L2
    bcc::DevBuf flush;
    BCC_CUDA(ctx, flush.ensure(kFlushBytes));
    bcc_opts opts{};
    opts.order = order;
    opts.use_graph = 1;
    cudaEvent_t e0, e1;
    BCC_CUDA(ctx, cudaEventCreate(&e0));
    BCC_CUDA(ctx, cudaEventCreate(&e1));
    const bool saved_prof = ctx->profiling;
    ctx->profiling = false;
    auto time_cfg = [&](const bcc::Tune& t, float& ms) -> bcc_status {
        ctx->tune = t;
        bcc_status s = run_check(ctx, robot, ctx->edges.as<float>(), num_edges, resolution, ctx->results.as<uint8_t>(),
                                 &opts, st);
        if (s != BCC_OK) return s;
        const bcc::GraphCache& G = ctx->graph[order == BCC_ORDER_LEARNED ? 1 : 0];
        const bool replay = G.exec && !ctx->counting && same_tune(G.tune, t);  // the graph just captured
        float reps[kTuneReps];
        for (int r = 0; r < kTuneReps; ++r) {
            BCC_CUDA(ctx, cudaMemsetAsync(flush.p, r, kFlushBytes, st));
            BCC_CUDA(ctx, cudaEventRecord(e0, st));
            if (replay) {
                BCC_CUDA(ctx, cudaGraphLaunch(G.exec, st));
            } else {  // no graph (work counters on): time the whole check
                s = run_check(ctx, robot, ctx->edges.as<float>(), num_edges, resolution, ctx->results.as<uint8_t>(),
                              &opts, st);
                if (s != BCC_OK) return s;
            }
            BCC_CUDA(ctx, cudaEventRecord(e1, st));
            BCC_CUDA(ctx, cudaEventSynchronize(e1));
            BCC_CUDA(ctx, cudaEventElapsedTime(&reps[r], e0, e1));
        }
        std::sort(reps, reps + kTuneReps);
        ms = reps[kTuneReps / 2];
        return BCC_OK;
    };
    bcc::Tune best = ctx->tune;
    float best_ms = 1e30f;
    bcc_status s = BCC_OK;
    auto keep = [&](const bcc::Tune& t) {
        float ms = 0;
        s = time_cfg(t, ms);
        if (s == BCC_OK && ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    };
    // Launch shape (edges per CTA x warps per CTA x persistent or not), and for
    // the learned order jointly with the queue threshold: the shape that suits
    // many queued pairs need not suit few, and a sweep of one at a time got
    // stuck on a worse pair (Fetch: 3 % off).
    const bool learned = order == BCC_ORDER_LEARNED && ctx->mlp.ready;
    const int tiles[4] = {32, 64, 128, 256};
    const int warps[2] = {4, 8};
    const int qmins[7] = {64, 128, 256, 512, 1024, 2048, 4096};
    const bcc::Tune base = best;
    // Launch shape first (for the learned order at a middle threshold with
    // one-warp finishes), then the learned order's threshold x finish mode at
    // that shape, then the shape once more at the chosen threshold and mode.
    // Lanes per walking pair: 16 only where the robot has the half-warp walk
    // (elsewhere it would time the 32-lane walk twice and could report 16).
    const int lanes[2] = {32, 16};
    const bcc::RobotOps* tops = bcc::robot_ops((int)robot);
    const int n_lanes = tops && tops->half_warp_walk ? 2 : 1;
    auto sweep_shape = [&](const bcc::Tune& from) {
        for (int ti = 0; ti < 4 && s == BCC_OK; ++ti)
            for (int wi = 0; wi < 2 && s == BCC_OK; ++wi)
                for (int pe = 0; pe < 2 && s == BCC_OK; ++pe)
                    for (int li = 0; li < n_lanes && s == BCC_OK; ++li) {
                        bcc::Tune t = from;
                        t.edges_per_cta = tiles[ti];
                        t.warps = warps[wi];
                        t.persistent = pe;
                        t.lanes = lanes[li];
                        keep(t);
                    }
    };
    bcc::Tune start = base;
    if (learned) {  // the inline order at one cluster while the shape is swept
        start.learned_mode = 0;
        start.clusters = 1;
    }
    sweep_shape(start);
    if (learned) {
        const bcc::Tune shape = best;
        const int ks[4] = {1, 4, 8, 16};
        for (int ki = 0; ki < 4 && s == BCC_OK; ++ki) {  // inline order: clusters
            bcc::Tune t = shape;
            t.learned_mode = 0;
            t.clusters = ks[ki];
            keep(t);
        }
        for (int qi = 0; qi < 7 && s == BCC_OK; ++qi)  // queued order: threshold x finish mode
            for (int sp = 0; sp < 2 && s == BCC_OK; ++sp) {
                bcc::Tune t = shape;
                t.learned_mode = 1;
                t.queue_min_items = qmins[qi];
                t.finish_split = sp;
                keep(t);
            }
        sweep_shape(best);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->profiling = saved_prof;
    best.tuned = true;
    ctx->tune = best;
    if (s != BCC_OK) return s;
    if (chosen) bcc_get_launch_config(ctx, chosen);
    return BCC_OK;
}

}  // extern "C"
