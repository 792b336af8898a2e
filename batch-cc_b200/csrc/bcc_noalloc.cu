// bcc_noalloc.cu -- the allocation-free check entry point.
//
// Some callers cannot allocate device memory: a planner that runs collision
// checks from a real-time control thread, where cudaMalloc's implicit device
// synchronisation and unbounded latency are not allowed; or a host framework
// that owns all device memory through its own pool and forbids other
// allocators.  bcc_check_noalloc serves them: it allocates nothing (no
// cudaMalloc/cudaFree, no allocating library call, no context object).  The
// caller passes every input and output in its own device memory; the working
// buffers live in the fixed file-scope arrays below.
//
// Limits: at most kMaxEdges edges and kMaxRows discretised samples (the sum of
// 32 n over the edges) per call; about 9 MB of device memory per GPU that loads
// the library, held until the process exits.
//
// All calls share these arrays, and each call leaves its contents behind;
// everything that must start at zero is cleared at the start of a call.  Calls
// that overlap on the GPU (two streams, two threads) race on the arrays: issue
// them one at a time.  The first call on each device does the per-device
// set-up (resolving the arrays' device addresses and uploading the robot
// tables).  No call can be made inside a stream capture: every call reads the
// sample count back to the host and synchronises the stream.  The set-up is
// done once per device for the life of the process, so a cudaDeviceReset after
// the first call is not supported (the robot tables would be gone while the
// set-up record says they are loaded).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/bcc.h"
#include "bcc_device.cuh"
#include "bcc_kernels.h"

namespace {

constexpr int kMaxEdges = 1024;
constexpr int kMaxRows = 4096;
constexpr int kNumSpheresMax = bcc::kMaxTableSpheres;  // widest sample-table row of any robot
constexpr int kGroupsMax = bcc::kMaxEnvGroups;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) int g_steps[kMaxEdges];
static __device__ __align__(256) int g_offs[kMaxEdges + 1];
static __device__ __align__(256) int g_edge_self[kMaxEdges];
static __device__ __align__(256) float4 g_swept[kMaxEdges * kGroupsMax * 2];
static_assert(kMaxRows % bcc::kMaxTableTile == 0, "the sample table holds whole tiles of rows");
static __device__ __align__(256) float4 g_table[kMaxRows * kNumSpheresMax];
static __device__ __align__(256) int g_row_edge[kMaxRows];
static __device__ __align__(256) int g_error[1];

struct Scratch {
    int* steps = nullptr;
    int* offs = nullptr;
    int* edge_self = nullptr;
    float4* swept = nullptr;
    float4* table = nullptr;
    int* row_edge = nullptr;
    int* error = nullptr;
    bool ready = false;
    bool tables[3] = {false, false, false};  // robot tables uploaded to this device
};

Scratch g_scratch[kMaxDevices];
std::mutex g_setup_mutex;

// Device addresses of the file-scope arrays (the host-side names are only
// stand-ins) and the robot's tables, once per device with that device current.
cudaError_t setup_device(int dev, const bcc::RobotOps* ops, Scratch*& out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    Scratch& s = g_scratch[dev];
    if (!s.ready) {
        cudaError_t e;
        if ((e = cudaGetSymbolAddress((void**)&s.steps, g_steps)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.offs, g_offs)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.edge_self, g_edge_self)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.swept, g_swept)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.table, g_table)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.row_edge, g_row_edge)) != cudaSuccess) return e;
        if ((e = cudaGetSymbolAddress((void**)&s.error, g_error)) != cudaSuccess) return e;
        s.ready = true;
    }
    if (!s.tables[ops->robot]) {
        cudaError_t e = ops->upload_tables();
        if (e != cudaSuccess) return e;
        s.tables[ops->robot] = true;
    }
    out = &s;
    return cudaSuccess;
}

}  // namespace

extern "C" bcc_status bcc_check_noalloc(bcc_robot robot, const float* d_records, const int32_t* d_env_offsets,
                                        int32_t num_envs, int32_t max_prims_per_env, const float* d_edges,
                                        int32_t num_edges, int32_t resolution, uint8_t* d_results, void* stream) {
    const bcc::RobotOps* ops = bcc::robot_ops((int)robot);
    if (!ops) return BCC_ERR_NOT_SUPPORTED;
    if (num_envs < 0 || num_edges < 0 || resolution <= 0 || max_prims_per_env < 0) return BCC_ERR_INVALID_ARGUMENT;
    if (num_edges > kMaxEdges) return BCC_ERR_LIMIT;  // more edges than the fixed working arrays hold
    if (max_prims_per_env > ops->max_prims) return BCC_ERR_LIMIT;
    if (bcc::records_smem_bytes(max_prims_per_env > 0 ? max_prims_per_env : 1, ops->num_env_groups,
                                bcc::kRecordsWarps) > 200 * 1024)
        return BCC_ERR_LIMIT;
    if (num_edges == 0 || num_envs == 0) return BCC_OK;
    if (!d_records && max_prims_per_env > 0) return BCC_ERR_INVALID_ARGUMENT;
    // The records are staged into shared memory by bulk copies, which need a
    // 16-byte-aligned source: refuse a misaligned pointer before any launch.
    if (max_prims_per_env > 0 && (reinterpret_cast<uintptr_t>(d_records) & 15u) != 0)
        return BCC_ERR_INVALID_ARGUMENT;
    if (!d_env_offsets || !d_edges || !d_results) return BCC_ERR_INVALID_ARGUMENT;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BCC_ERR_CUDA;
    Scratch* s = nullptr;
    if (setup_device(dev, ops, s) != cudaSuccess) return BCC_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Stale contents from the previous call: clear what must start at zero (the
    // per-edge self-collision flags are cleared by the prep stage itself).
    if (cudaMemsetAsync(s->error, 0, sizeof(int), st) != cudaSuccess) return BCC_ERR_CUDA;

    bcc::PipelineArgs a{};
    a.d_edges = d_edges;
    a.num_edges = num_edges;
    a.resolution = resolution;
    a.steps = s->steps;
    a.offs = s->offs;
    a.edge_self = s->edge_self;
    a.swept = s->swept;
    a.table = s->table;
    a.row_edge = s->row_edge;
    if (ops->steps(a, st) != cudaSuccess) return BCC_ERR_CUDA;
    int total = 0;
    if (cudaMemcpyAsync(&total, s->offs + num_edges, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return BCC_ERR_CUDA;
    if (total < 0 || total > kMaxRows) return BCC_ERR_LIMIT;  // the edges need more samples than the arrays hold
    a.total_rows = total;
    if (ops->prep(a, st) != cudaSuccess) return BCC_ERR_CUDA;

    bcc::RecordsParams P{};
    P.records = reinterpret_cast<const float4*>(d_records);
    P.env_off = d_env_offsets;
    P.num_envs = num_envs;
    P.num_edges = num_edges;
    P.max_prims = max_prims_per_env > 0 ? max_prims_per_env : 1;
    P.edges_per_cta = 64;
    P.steps = s->steps;
    P.offs = s->offs;
    P.table = s->table;
    P.swept = s->swept;
    P.edge_self = s->edge_self;
    P.results = d_results;
    P.error_flag = s->error;
    if (ops->check_records(P, st) != cudaSuccess) return BCC_ERR_CUDA;
    int flag = 0;
    if (cudaMemcpyAsync(&flag, s->error, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return BCC_ERR_CUDA;
    if (flag & 2) return BCC_ERR_INVALID_ARGUMENT;  // an environment exceeds max_prims_per_env
    return flag ? BCC_ERR_TIMEOUT : BCC_OK;
}
