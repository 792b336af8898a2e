// bcc_ctx.h -- the checker context (internal; the C ABI sees an opaque bcc_ctx).
#pragma once

#include <algorithm>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace bcc {

// Device buffer grown on demand and reused across calls.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        const size_t want = std::max(bytes, cap * 3 / 2);
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// State of the collision-likelihood MLP (weights, optimiser, scratch).
struct MlpState {
    bool ready = false;      // weights uploaded
    DevBuf params;           // FP32 master parameters (kMlpParams floats)
    DevBuf grads;            // FP32 gradients
    DevBuf adam_m, adam_v;   // Adam moments
    DevBuf images;           // BF16 core-matrix images of W1^T, W2^T, W3^T
    DevBuf acts;             // training activations
    DevBuf x, y, logits;     // per-call inputs / outputs
    DevBuf lab;              // learned-order population: per-sample verdicts (8 per row)
    DevBuf x2, y2, perm;     // shuffled training rows and their permutation
    long long step = 0;      // Adam step count
};

// Launch configuration of the environment check (set by bcc_autotune).
struct Tune {
    int edges_per_cta = 128;
    int warps = 8;
    int persistent = 1;
    int queue_min_items = 128;
    int finish_split = 0;    // learned order, queued: 1 = split each queued pair over a CTA's warps
    int learned_mode = 0;    // learned order: 0 = inline (per-cluster scores), 1 = queued (per-pair scores)
    int clusters = 1;        // learned order, inline: environment clusters scored per edge
    int lanes = 32;          // lanes per walking pair in the plain-order walk: 32 or 16 (half-warps)
    bool tuned = false;
};

// A captured launch sequence (everything after the discretisation) and the
// inputs it was captured for.
struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    const void* edges = nullptr;
    void* results = nullptr;
    cudaStream_t stream = nullptr;
    int num_edges = -1, resolution = -1, total_rows = -1, order = -1, robot = -1, row_cap = -1;
    long long env_version = -1;
    Tune tune;
    ~GraphCache() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

}  // namespace bcc

struct bcc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t capture_stream = nullptr;  // private stream for CUDA-graph capture
    std::string err;
    bool tables[3] = {false, false, false};
    // environment arena
    int num_envs = -1;
    int max_prims = 0;
    size_t blob_smem = 0;

    bcc::DevBuf blobs, env_hdr;
    // per-call buffers
    bcc::DevBuf edges, steps, offs, table, row_edge, edge_self, swept, results, error_flag;
    int* h_total = nullptr;  // pinned readback of the sample-row total
    bool profiling = false;
    bool counting = false;
    bcc::DevBuf counters;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    // learned proposal
    bcc::MlpState mlp;
    bcc::DevBuf edge_tri;    // [E][groups] packed slab ranges of each group's swept box
    bcc::DevBuf grid_bounds; // [3][kGridSlabs + 1] slab boundaries of the uploaded set's cull grid
    bcc::DevBuf env_code;    // [num_envs][32] environment encodings
    bool env_code_ready = false;
    // inline learned order: environment clusters (k-means over the codes)
    bcc::DevBuf env_cluster; // [num_envs] cluster id
    bcc::DevBuf centroids;   // [K][32] cluster centroid codes
    int cluster_k = 0;       // K of the current clustering, 0 = none
    bcc::DevBuf perms;       // [K][edges][32] per-check lane-block permutations
    bcc::DevBuf q_head, q_pairs, q_rows;   // learned-order queue of undecided pairs
    const int* learned_rows_dev = nullptr; // queue head of the last learned check (entries << 32 | rows)
    int learned_row_cap = 0;
    bool last_learned_inline = false;      // the last learned check used the inline order
    long long last_inline_rows = 0;        // its (cluster, segment) rows
    int learned_q_cap = 0;
    bcc::Tune tune;                        // launch configuration (autotuned or default)
    bcc::DevBuf work_counter;              // persistent-kernel work queue head
    long long env_version = 0;             // bumped by every upload (graph cache key)
    bcc::GraphCache graph[2];              // per order (plain, learned)
};
