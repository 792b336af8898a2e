/*
 * bcc.h -- C ABI of the B200 batch edge collision checker.
 *
 * Drop-in boundary for the reference entry point
 *   template <typename Robot> void batch_cc::batch_cc(
 *       std::vector<ppln::collision::Environment<float>>& h_envs,
 *       std::vector<std::array<typename Robot::Configuration, 2>>& edges,
 *       int resolution, std::vector<bool>& results);
 * declared at src/batch_cc.hh:4-6 and defined at src/batch_cc.cu:244-338.
 *
 * Every entry point takes plain pointers and sizes (no C++ or torch types) and
 * returns a bcc_status.  Verdicts keep the reference's meaning and layout:
 * results[edge * num_envs + env] = 1 when the discretised edge is IN COLLISION
 * in that environment (src/batch_cc.cu:130-132), 0 when it is free.
 */
#ifndef BCC_H
#define BCC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bcc_status {
    BCC_OK = 0,
    BCC_ERR_INVALID_ARGUMENT = 1, /* null pointer with a positive count, bad size, unknown robot */
    BCC_ERR_CUDA = 2,             /* a CUDA runtime call failed; see bcc_last_error */
    BCC_ERR_NO_ENVS = 3,          /* bcc_check before any bcc_upload_envs */
    BCC_ERR_TIMEOUT = 4,          /* a bounded device-side wait gave up */
    BCC_ERR_NOT_SUPPORTED = 5,    /* option or robot not available in this build */
    BCC_ERR_LIMIT = 6             /* a size exceeds a documented maximum */
} bcc_status;

typedef enum bcc_robot {
    BCC_ROBOT_PANDA = 0,  /* src/Robots.hh:10-64, 7 DOF */
    BCC_ROBOT_FETCH = 1,  /* src/Robots.hh:66-120, 8 DOF */
    BCC_ROBOT_BAXTER = 2  /* src/Robots.hh:122-188, 14 DOF */
} bcc_robot;

/*
 * Environments in structure-of-arrays form: per-environment primitive counts,
 * and the records of all environments concatenated in environment order.
 * Record layouts follow the reference shapes (src/collision/shapes.hh) without
 * their std::string header:
 *   sphere   [4]  x y z r                                   (shapes.hh:226-245)
 *   capsule  [8]  x1 y1 z1 xv yv zv r rdv  (rdv = 1/|v|^2)  (shapes.hh:131-222)
 *   cuboid   [15] x y z  a1x a1y a1z  a2x a2y a2z  a3x a3y a3z  h1 h2 h3
 *                                                           (shapes.hh:30-126)
 * z_capsules / z_cuboids are the axis-aligned variants tested with the
 * reference's z-aligned predicates (src/utils.cuh:138-156, :187-210).
 * Cylinders are accepted but, exactly as in the reference device scan
 * (src/utils.cuh:213-245), never tested: the reference drivers pass
 * cylinders as capsules.
 * A null count array means zero primitives of that kind in every environment.
 */
typedef struct bcc_env_soa {
    int32_t num_envs;
    const uint32_t* num_spheres;
    const uint32_t* num_capsules;
    const uint32_t* num_z_capsules;
    const uint32_t* num_cuboids;
    const uint32_t* num_z_cuboids;
    const uint32_t* num_cylinders;
    const float* spheres;
    const float* capsules;
    const float* z_capsules;
    const float* cuboids;
    const float* z_cuboids;
    const float* cylinders;
} bcc_env_soa;

/* Sample-check order inside each (environment, edge) pair. */
typedef enum bcc_order {
    BCC_ORDER_PLAIN = 0,   /* ascending sample index */
    BCC_ORDER_LEARNED = 1  /* descending collision likelihood from the proposal MLP */
} bcc_order;

typedef struct bcc_opts {
    int32_t order;         /* bcc_order */
    int32_t use_graph;     /* 1: replay a captured CUDA graph of the launch sequence */
    int32_t tile_override; /* 0: autotuned tile; >0: force a tile id (tuning/tests) */
    int32_t learned_row_cap; /* learned order: 0 = default budget of MLP rows (segments scored) per
                              * check, >0 = at most this many; pairs beyond it keep the plain order */
} bcc_opts;

typedef struct bcc_ctx bcc_ctx;

/* Context lifetime.  A context owns device buffers that persist across calls. */
bcc_status bcc_create(bcc_ctx** out, int device);
void bcc_destroy(bcc_ctx* ctx);
const char* bcc_last_error(const bcc_ctx* ctx);

/*
 * Upload (replace) the environment set.  Replaces the reference's per-env
 * setup_environment_on_device / cleanup_environment_on_device
 * (src/batch_cc.cu:135-240) with one packed device arena.  Rejects a positive
 * count with a null record pointer, like ensure_ptr_count_consistent
 * (src/batch_cc.cu:45-56).
 */
bcc_status bcc_upload_envs(bcc_ctx* ctx, const bcc_env_soa* envs);

/*
 * Check every (environment, edge) pair.  edges: host array float[num_edges][2][dof]
 * (start, end), the reference's layout (src/batch_cc.cu:292-295).  results: host
 * array of num_envs * num_edges bytes, edge-major.  resolution: the reference's
 * step multiplier (32 in its drivers, scripts/batch_cc_mbm.cpp:184).
 * Synchronous: returns after the verdicts are in host memory.
 */
bcc_status bcc_check(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges,
                     int32_t resolution, uint8_t* results, const bcc_opts* opts);

/*
 * Device-resident variant: edges and results are device pointers; the call is
 * stream-ordered on `stream` (a cudaStream_t, 0 = legacy default stream) and
 * returns without synchronising.
 */
bcc_status bcc_check_device(bcc_ctx* ctx, bcc_robot robot, const float* d_edges,
                            int32_t num_edges, int32_t resolution, uint8_t* d_results,
                            const bcc_opts* opts, void* stream);

/*
 * Host-only helper (no CUDA call): pack an environment set into the device
 * arena format -- one 80-byte "rounded box" record per primitive (20 floats:
 * centre xyz, rounding radius; axis1 xyz, h1; axis2 xyz, h2; axis3 xyz, h3;
 * cull AABB half-size xyz, 0) and env_offsets[num_envs + 1] (first record of
 * each environment).  Pass records = NULL to query the record count through
 * *num_records.  Performs the same validation as bcc_upload_envs.
 */
bcc_status bcc_pack_envs(const bcc_env_soa* envs, float* records, int32_t* env_offsets,
                         int64_t* num_records, int32_t* max_prims_per_env);

/*
 * Stage timing.  With profiling on, every check records CUDA events around its
 * stages on the launch stream; bcc_stage_times returns the last check's device
 * milliseconds (after the stream has been synchronised by the caller):
 *   [0] discretisation + sample offsets  [1] forward kinematics table
 *   [2] self-collision                    [3] swept cull volumes
 *   [4] environment check (the dominant kernel)
 * Returns the number of stages written, or -1.
 */
bcc_status bcc_set_profiling(bcc_ctx* ctx, int32_t on);
int32_t bcc_stage_times(bcc_ctx* ctx, float* ms, int32_t max_stages);

/*
 * Work counters of the last check, when profiling was switched on with bit 1
 * set (bcc_set_profiling(ctx, 3)): [0] pairs walked, [1] candidate
 * (primitive, link) pairs after the cull, [2] walk steps (32 items, or 16
 * with 16 lanes per walking pair), [3] steps with a gate hit, [4] leaf steps,
 * [5] colliding pairs.  Diagnostics only: counting
 * adds atomics to the check kernel.  Returns the number written, or -1.
 */
int32_t bcc_work_counters(bcc_ctx* ctx, uint64_t* out, int32_t max_counters);

/*
 * Allocation-free check.  No counterpart in the reference: this entry point
 * exists for callers that cannot allocate device memory -- for example a
 * planner checking edges from a real-time control thread, where cudaMalloc's
 * implicit device synchronisation and unbounded latency are not allowed, or a
 * host framework that owns all device memory through its own pool.  It makes
 * no cudaMalloc/cudaFree or other allocating call and needs no bcc_ctx; its
 * working buffers are fixed arrays inside the library (about 9 MB on every GPU
 * that loads it, kept until the process exits).
 *   d_records / d_env_offsets: device copies of bcc_pack_envs' output
 *     (records 16-byte aligned); max_prims_per_env: its max_prims_per_env.
 *   d_edges: device float[num_edges][2][dof]; d_results: device
 *     uint8[num_edges][num_envs], same meaning and layout as bcc_check.
 * Limits: num_edges <= 1024 and at most 4096 discretised samples per call
 * (sum over edges of 32 n); beyond either the call returns BCC_ERR_LIMIT
 * without checking anything.  d_records must be 16-byte aligned (bulk copies
 * stage it); a misaligned pointer returns BCC_ERR_INVALID_ARGUMENT before any
 * launch.  Synchronous on `stream`: every call reads the sample count back and
 * synchronises, so no call can be made inside a stream capture.  The first call
 * on a device sets that device up for the life of the process (resolves the
 * arrays' addresses, uploads the robot tables); a cudaDeviceReset after it is
 * not supported.  Every call reuses the same arrays, so calls that overlap on
 * the GPU race; issue them one at a time.
 */
bcc_status bcc_check_noalloc(bcc_robot robot, const float* d_records, const int32_t* d_env_offsets,
                             int32_t num_envs, int32_t max_prims_per_env, const float* d_edges,
                             int32_t num_edges, int32_t resolution, uint8_t* d_results, void* stream);

/*
 * Collision-likelihood MLP of the learned check order (no reference
 * counterpart; it proposes the order in which the exact check visits an
 * edge's samples).  Input row: 48 BF16 features (the robot's joints
 * normalised to [-1, 1] by the joint limits, the 32-value environment code,
 * zeros, the sample's position along its edge in [-1, 1] as feature 46;
 * feature 47 is the bias input the forward kernel reads as 1); 3 hidden
 * layers of 128 (ReLU); output: one logit (collision likelihood).  Parameters are FP32 masters, flat, in the order
 * W1[48][128], b1[128], W2[128][128], b2[128], W3[128][128], b3[128], w4[128],
 * b4[1]; the kernels use BF16 copies on tcgen05 tensor cores with FP32
 * accumulation.
 */
int32_t bcc_mlp_num_params(void);
bcc_status bcc_mlp_set_params(bcc_ctx* ctx, const float* params, int32_t num_params);
bcc_status bcc_mlp_get_params(bcc_ctx* ctx, float* params, int32_t num_params);
/* d_x: device BF16 [rows][48]; d_logits: device FP32 [rows]; stream-ordered. */
bcc_status bcc_mlp_forward(bcc_ctx* ctx, const void* d_x_bf16, int32_t rows, float* d_logits, void* stream);
/* Gradient of the mean binary cross-entropy over `rows` labelled rows (labels
 * 0/1, device uint8) with respect to every parameter, by the tensor-core
 * training kernel; h_grads: host FP32 [num_params] (may be NULL), h_loss: host
 * summed loss (may be NULL). */
bcc_status bcc_mlp_gradients(bcc_ctx* ctx, const void* d_x_bf16, const uint8_t* d_labels, int32_t rows,
                             float* h_grads, float* h_loss);
/*
 * Train on checker-labelled samples: num_samples (environment, edge, sample)
 * triples drawn (seeded) from the uploaded environments and the given host
 * edges; label = the sample's environment collision by this library's check.
 * Adam, `epochs` passes in batches of `batch` rows.  h_epoch_loss[epochs]: mean
 * loss per epoch (may be NULL); h_positive_fraction: label balance (may be NULL).
 */
bcc_status bcc_mlp_train(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges, int32_t resolution,
                         int64_t num_samples, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                         float* h_epoch_loss, float* h_positive_fraction);
/*
 * Train on the population the learned order acts on: the (environment, edge)
 * pairs that the probe -- the plain walk of each pair's rank 0, its first
 * sample -- leaves undecided with at least queue_min_items (sample, pair)
 * items to go, over the uploaded environments and the given host edges.  One
 * row per segment of such a pair (features at the segment's scored sample, its
 * last one), labelled by this library's exact check of that sample; a seeded
 * shuffle of at most num_samples of them, Adam, `epochs` passes in batches of
 * `batch` rows.  h_rows (may be NULL) receives the rows used; fewer than one
 * batch returns BCC_ERR_INVALID_ARGUMENT.
 */
bcc_status bcc_mlp_train_queued(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges,
                                int32_t resolution, int32_t queue_min_items, int64_t num_samples, int32_t epochs,
                                int32_t batch, float lr, uint64_t seed, float* h_epoch_loss,
                                float* h_positive_fraction, int64_t* h_rows);
/*
 * Ranking quality of the current network on the learned order's population
 * (the pairs queued at queue_min_items, as for bcc_mlp_train_queued), judged
 * by this library's exact per-sample checks.  h_metrics[0..12]:
 *   [0] queued pairs, [1] scored segments, [2] colliding fraction of the queued
 *   pairs, [3] colliding fraction of the scored samples, [4] AUC of the segment
 *   scores against the scored samples' verdicts; sample ranks walked after the
 *   probe until the first hit, mean over the colliding queued pairs, in the
 *   [5] plain order (reference ranks 1, 2, ...), [6] learned order (segments by
 *   descending score, each from its last sample), [7] perfect order (1);
 *   [8..10] the same means over all queued pairs (collision-free pairs walk
 *   all their samples); [11] share of the perfect order's saving over the plain
 *   order that the learned order realises on the colliding pairs; [12]
 *   misprediction rate of the scored samples (sign of the logit vs verdict).
 */
bcc_status bcc_mlp_rank_metrics(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges,
                                int32_t resolution, int32_t queue_min_items, double* h_metrics,
                                int32_t max_metrics);
/* Held-out metrics on fresh samples: [0] mean BCE, [1] misprediction rate (sign
 * of the logit vs the checker's verdict), [2] false-positive rate, [3]
 * false-negative rate, [4] positive fraction. */
bcc_status bcc_mlp_evaluate(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges, int32_t resolution,
                            int64_t num_samples, uint64_t seed, float* h_metrics);
/* The 32-value environment code of every uploaded environment (the MLP's
 * environment features), h_code: host float[num_envs][32], num_envs as
 * uploaded.  [0..2] counts of sphere-, capsule- and box-like primitives / 64,
 * [3] total / 64; [4 + 3a + k] for anchor a = (+-0.35, +-0.35, 0.3 | 0.8) m
 * (bit 0: x, bit 1: y, bit 2: z) the signed distance to the nearest primitive
 * of kind k, clamped to [-0.5, 1.5] m (1.5 without one); [28..30] mean centre,
 * [31] mean rounding radius + half-extent sum. */
bcc_status bcc_env_code(bcc_ctx* ctx, float* h_code, int32_t num_envs);
/* MLP rows (segments) scored by the last learned-order check. */
int64_t bcc_last_learned_rows(const bcc_ctx* ctx);
/* (environment, edge) pairs the last learned-order check queued for the MLP
 * order (the others were decided, or walked on, in plain order by the probe). */
int64_t bcc_last_learned_pairs(const bcc_ctx* ctx);
/* One Adam step (learning rate lr) on the gradient of the batch. */
bcc_status bcc_mlp_train_step(bcc_ctx* ctx, const void* d_x_bf16, const uint8_t* d_labels, int32_t rows,
                              float lr, float* h_loss);

/* Diagnostics: FP32 FMA-pipe throughput of `device` in TFLOP/s, measured by a
 * short probe kernel (the roofline denominator of the scalar-FP32 checker). */
bcc_status bcc_measure_fp32_peak(int32_t device, double* tflops);

/*
 * Launch configuration of the environment check, BCC_LAUNCH_CONFIG_LEN values:
 * cfg[0] edges per CTA, cfg[1] warps per CTA (1, 2, 4, 8; lowered
 * automatically when an environment's shared-memory footprint needs it),
 * cfg[2] 1 = persistent kernel pulling (environment, edge tile) work items
 * from an atomic queue, 0 = one CTA per item, cfg[3] learned order: a pair is
 * scored by the MLP only when at least this many (sample, pair) items remain
 * once its rank 0 (first sample) is walked, cfg[4] learned order: 1 = each
 * queued pair's walk split over a CTA's warps, 0 = one warp per queued pair,
 * cfg[5] learned order: 0 = inline (every pair walks its first sample, then
 * its other samples in the order the MLP scored for its environment's
 * cluster, in one pass), 1 = queued (pairs left undecided by a plain probe of
 * their first sample are scored per pair and finished in a second pass),
 * cfg[6] inline order: environment clusters, 1..64 (k-means over the
 * environment codes; the MLP scores each edge's segments once per cluster),
 * cfg[7] lanes per walking pair in the plain-order walk: 32 (a whole warp) or
 * 16 (the warp's halves walk two pairs at once, 16 items a step each; robots
 * whose leaves lie inside their bounds, otherwise 32 is used).
 */
#define BCC_LAUNCH_CONFIG_LEN 8
bcc_status bcc_get_launch_config(const bcc_ctx* ctx, int32_t* cfg);
bcc_status bcc_set_launch_config(bcc_ctx* ctx, const int32_t* cfg);
/*
 * Autotuner: times candidate configurations (edges per CTA 32..256, 4 or 8
 * warps, persistent or not, 32 or 16 lanes per walking pair; for the learned
 * order also the inline order's
 * cluster count and the queued order's threshold 64..4096 items and finish
 * mode) on the given host edges against the
 * uploaded environments, timing graph replays, and keeps the fastest in the
 * context; chosen[BCC_LAUNCH_CONFIG_LEN] receives it (may be NULL).
 * order: bcc_order.
 */
bcc_status bcc_autotune(bcc_ctx* ctx, bcc_robot robot, const float* edges, int32_t num_edges, int32_t resolution,
                        int32_t order, int32_t* chosen);

/* Number of samples the reference discretisation checks for one edge
 * (32 * max(ceil(|end - start|_2 / 31 * resolution), 1), src/batch_cc.cu:103-116). */
int32_t bcc_edge_samples(const float* start, const float* end, int32_t dof, int32_t resolution);

/* Robot degrees of freedom (7, 8, 14), or -1 for an unknown robot. */
int32_t bcc_robot_dof(bcc_robot robot);

#ifdef __cplusplus
}
#endif

#endif /* BCC_H */
