// bcc_kernels.h -- host-visible launch interface of the checker kernels.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace bcc {

// Cull grid of an environment set: kGridSlabs slabs per axis (boundaries at
// quantiles of the primitives' centres); per environment and slab range
// [i0, i1] (triangular index) a bit mask of the primitives whose AABB meets
// that range.
constexpr int kGridSlabs = 32;
constexpr int kGridTri = kGridSlabs * (kGridSlabs + 1) / 2;

__host__ __device__ __forceinline__ int tri_index(int i0, int i1) {
    return i0 * kGridSlabs - (i0 * (i0 - 1)) / 2 + (i1 - i0);
}

struct CheckParams {
    const float4* blobs;     // per env: [np][5] rounded-box records, then 3 x kGridTri x W masks
    const float4* env_hdr;   // [num_envs][2]: (grid origin xyz, blob offset in float4s),
                             //                 (1/slab width xyz, np | W << 16)
    int num_envs;
    int num_edges;
    int max_prims;           // max primitives of one env (pair-list sizing)
    size_t blob_smem;        // bytes of the largest env's records (16-byte multiple)
    int pairs_per_warp;
    int edges_per_cta;
    const int* steps;        // [E] n per edge
    const int* offs;         // [E + 1] first sample row of each edge
    const float4* table;     // [rows][num_spheres] sphere centres + radius
    const float4* swept;     // [E][groups][2] cull AABB centre / half-size
    const int* edge_tri;     // [E][groups] slab ranges on the set's grid (tx | ty << 10 | tz << 20), -1 = none
    const int* edge_self;    // [E] 1 when some sample self-collides
    uint8_t* results;        // [E][num_envs]
    int* error_flag;         // set when a bounded wait gives up
    unsigned long long* counters;  // null, or kNumCounters work counters (diagnostics)
    // Learned order (probe and finish); unused in plain mode.
    unsigned long long* q_head;  // queue entries handed out << 32 | MLP rows handed out
    int2* q_pairs;           // [q_cap] queued (edge, environment)
    int* q_rows;             // [q_cap] first MLP row of the entry, -1 = none (the probe walked on)
    int q_cap;               // capacity of the queue arrays
    int row_cap;             // capacity of the MLP row buffers
    const float* logits;     // [row_cap] segment scores (finish)
    int queue_min_items;     // probe: queue only pairs with at least this many items left
    int* finish_counter;     // next queue entry for the finish kernel
    int finish_split;        // 1: each queued pair split over a CTA's warps, 0: one warp per pair
    int persistent;          // 1: persistent kernel pulling work items from work_counter
    int* work_counter;
    // Inline learned order (mode 4): per (cluster, edge) segment permutations.
    const int* env_cluster;  // [num_envs] cluster of each environment
    const uint8_t* perms;    // [K][num_edges][32] lane block at each rank of a round
    int total_segs;          // offs[E] / kSegment
};

// Samples per learned-order segment: the MLP scores each run of 8 consecutive
// samples at its last sample, where the walk of the segment starts; an edge
// with step count n has 4 n segments.
constexpr int kSegment = 8;
constexpr int kMaxSegments = 64;  // edges with more segments keep the plain order

// Work counters of the environment check (diagnostics, off by default):
// pairs walked, candidate (primitive, link) pairs, 32-item chunks, gate steps
// with a hit, leaf steps, colliding pairs.
constexpr int kNumCounters = 6;

struct PipelineArgs {
    const float* d_edges;    // [E][2][dof]
    int num_edges;
    int resolution;
    int* steps;              // [E]
    int* offs;               // [E + 1]
    int total_rows;          // offs[E], read back after the scan
    float4* table;           // [total_rows][num_spheres]
    int* row_edge;           // [total_rows]
    const uint8_t* fk_perm;  // null, or [E][32] lane-block permutation the FK table is written in
    int* edge_self;          // [E]
    float4* swept;           // [E][groups][2]
    int* edge_tri;           // [E][groups], null = not needed (records check)
    const float* grid_bounds;  // [3][kGridSlabs + 1] cull-grid slab boundaries of the environment set
    const float4* blobs;
    const float4* env_hdr;
    int num_envs;
    int max_prims;
    size_t blob_smem;
    int edges_per_cta;
    int warps;               // warps per check CTA (8, 4, 2 or 1)
    uint8_t* d_results;
    int* error_flag;
    cudaEvent_t* stage_events;  // null, or 6 events bracketing the 5 stages
    unsigned long long* counters;
    int mode;                // 0 plain, 1 probe (rank 0, queue the rest), 2 finish (learned order),
                             // 4 inline learned order
    unsigned long long* q_head;
    int2* q_pairs;
    int* q_rows;
    int q_cap;
    int row_cap;
    const float* logits;
    int queue_min_items;
    int* finish_counter;
    int finish_split;
    int persistent;
    int* work_counter;
    const int* env_cluster;
    const uint8_t* perms;
    int total_segs;
};

// Environment check from host-packed records (bcc_pack_envs format), exact
// AABB cull; used by the allocation-free entry point.
struct RecordsParams {
    const float4* records;   // [total prims][5] rounded-box records
    const int* env_off;      // [num_envs + 1]
    int num_envs;
    int num_edges;
    int max_prims;
    int pairs_per_warp;
    int edges_per_cta;
    const int* steps;
    const int* offs;
    const float4* table;
    const float4* swept;
    const int* edge_self;
    uint8_t* results;
    int* error_flag;
};

// Limits every robot model must respect (checked at compile time by the
// robot's translation unit): link groups (one cull lane each) and sample-table
// row width.
constexpr int kMaxEnvGroups = 32;
constexpr int kMaxTableSpheres = 128;
constexpr int kRecordsWarps = 4;  // warps per CTA of the records check kernel
// Entries of a warp's (primitive, link) pair list in shared memory; a pair with
// more candidates is walked in segments of this many.
constexpr int kPairCap = 1024;

// One robot's pipeline, instantiated in its own translation unit
// (bcc_robot_<name>.cu) from the templates of bcc_pipeline.cuh.
struct RobotOps {
    int robot;               // bcc_robot id
    int dof;
    int num_spheres;         // sample-table row width (float4 per sample)
    int num_env_groups;
    int max_prims;           // primitives per environment the pair packing allows
    bool half_warp_walk;     // the 16-lane walk exists (no overhang, grouped cull); else lanes 16 walks as 32
    cudaError_t (*upload_tables)();  // robot tables -> __constant__ of the current device
    // Stage 1: steps + sample offsets (total rows land in offs[E]).
    cudaError_t (*steps)(const PipelineArgs& a, cudaStream_t st);
    // Stage 2: FK table, self-collision, swept volumes, environment check.
    cudaError_t (*check)(const PipelineArgs& a, cudaStream_t st);
    // FK table, self-collision and swept volumes only.
    cudaError_t (*prep)(const PipelineArgs& a, cudaStream_t st);
    // Environment check only, in a.mode.
    cudaError_t (*check_mode)(const PipelineArgs& a, cudaStream_t st);
    cudaError_t (*queue_features)(const PipelineArgs& a, const float* env_code, uint16_t* x, int grid,
                                  cudaStream_t st);
    cudaError_t (*training_rows)(const PipelineArgs& a, const float* env_code, long long rows,
                                 unsigned long long seed, uint16_t* x, uint8_t* y, cudaStream_t st);
    cudaError_t (*check_records)(RecordsParams P, cudaStream_t st);
    // Learned-order population: per-sample environment verdicts of the queued
    // pairs (lab, 8 per MLP row) and of each segment's scored sample (y).
    cudaError_t (*queue_labels)(const PipelineArgs& a, uint8_t* lab, uint8_t* y, int grid, cudaStream_t st);
    // Inline learned order: MLP feature rows of every (cluster, segment) and,
    // from their scores (a.logits), the per-(cluster, edge) 32-block permutations.
    cudaError_t (*cluster_features)(const PipelineArgs& a, const float* centroids, int K, uint16_t* x,
                                    cudaStream_t st);
    cudaError_t (*cluster_perms)(const PipelineArgs& a, int K, uint8_t* perms, cudaStream_t st);
};

// null for a robot this library was not built with.
const RobotOps* robot_ops(int robot);

// Robot-independent kernels (bcc_kernels.cu).
cudaError_t launch_scan(const int* steps, int E, int* offs, cudaStream_t st);
cudaError_t launch_env_encode(const float4* blobs, const float4* env_hdr, int num_envs, float* code, cudaStream_t st);
// Row gather for training: x2[i] = x[perm[i]] (kMlpIn BF16 values), y2[i] = y[perm[i]].
cudaError_t launch_gather_rows(const uint16_t* x, const uint8_t* y, const int* perm, int rows, uint16_t* x2,
                               uint8_t* y2, cudaStream_t st);
size_t check_smem_bytes(int max_prims, int groups, size_t blob_smem, int warps);
size_t records_smem_bytes(int max_prims, int groups, int warps);

inline CheckParams params_of(const PipelineArgs& a) {
    CheckParams P{};
    P.blobs = a.blobs;
    P.env_hdr = a.env_hdr;
    P.num_envs = a.num_envs;
    P.num_edges = a.num_edges;
    P.max_prims = a.max_prims;
    P.blob_smem = a.blob_smem;
    P.edges_per_cta = a.edges_per_cta;
    P.steps = a.steps;
    P.offs = a.offs;
    P.table = a.table;
    P.swept = a.swept;
    P.edge_tri = a.edge_tri;
    P.edge_self = a.edge_self;
    P.results = a.d_results;
    P.error_flag = a.error_flag;
    P.counters = a.counters;
    P.q_head = a.q_head;
    P.q_pairs = a.q_pairs;
    P.q_rows = a.q_rows;
    P.q_cap = a.q_cap;
    P.row_cap = a.row_cap;
    P.logits = a.logits;
    P.queue_min_items = a.queue_min_items;
    P.finish_counter = a.finish_counter;
    P.finish_split = a.finish_split;
    P.persistent = a.persistent;
    P.work_counter = a.work_counter;
    P.env_cluster = a.env_cluster;
    P.perms = a.perms;
    P.total_segs = a.total_segs;
    return P;
}

}  // namespace bcc
