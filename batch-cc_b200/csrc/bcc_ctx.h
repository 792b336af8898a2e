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
    long long step = 0;      // Adam step count
};

}  // namespace bcc

struct bcc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
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
    bcc::DevBuf env_code;    // [num_envs][32] environment encodings
    bool env_code_ready = false;
    bcc::DevBuf q_count, q_edges, q_rows;  // learned-order queue of undecided pairs
    long long last_learned_rows = 0;       // MLP rows scored by the last learned check
    int queue_min_items = 128;             // learned order: remaining items that justify scoring
};
