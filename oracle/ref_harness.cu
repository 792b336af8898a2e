// ref_harness.cu -- C entry points around the reference's own CUDA path.
//
// TEST INFRASTRUCTURE ONLY (the parity checker and the reference timing arm).
// This translation unit #includes the reference's src/batch_cc.cu unmodified
// (compiled for sm_100a from the reference tree by oracle/Makefile, target
// `ref`) and exposes:
//   ref_check          -- batch_cc::batch_cc<Robot>, the reference public API
//                         (src/batch_cc.hh:4-6), on environments rebuilt with
//                         the reference shape constructors;
//   ref_time           -- the reference kernel batch_cc_kernel<Robot>
//                         (src/batch_cc.cu:74-133) on environments placed by the
//                         reference's setup_environment_on_device, timed with
//                         CUDA events;
//   ref_probe_samples  -- batch_cc_kernel instantiated with a probe robot whose
//                         fkcc records every configuration the kernel checks: the
//                         reference's exact discretisation, as golden vectors.
// Robot = Panda, Fetch or Baxter.  The reference's Fetch and Baxter check
// functions (fkcc<Fetch> src/utils.cuh:10382, fkcc<Baxter> :24994) have the
// three-argument signature while batch_cc_kernel calls the five-argument one,
// and their batch_cc instantiations are commented out (src/batch_cc.cu:341-342);
// this file adds five-argument specialisations that forward to the reference's
// own three-argument functions, and the two instantiations, without touching
// the reference sources.
// Headers the reference received transitively through Eigen (std::memcpy).
#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <cstring>

#include "src/batch_cc.cu"

#include "../include/bcc.h"

namespace {

using ppln::collision::Capsule;
using ppln::collision::Cuboid;
using ppln::collision::Environment;
using ppln::collision::Sphere;

struct ProbeRobot {
    static constexpr auto name = "probe";
    static constexpr auto dimension = 7;
    using Configuration = std::array<float, dimension>;
};

__device__ float* g_probe_out;   // [E][32][kProbeRounds][7]
__device__ int* g_probe_count;   // [E][32]
constexpr int kProbeRounds = 16;

// Keeps stdout clean while the reference prints its timing lines.
struct QuietStdout {
    int saved = -1;
    explicit QuietStdout(bool on) {
        if (!on) return;
        fflush(stdout);
        std::cout.flush();
        saved = dup(1);
        dup2(2, 1);
    }
    ~QuietStdout() {
        if (saved < 0) return;
        fflush(stdout);
        std::cout.flush();
        dup2(saved, 1);
        close(saved);
    }
};

std::vector<Environment<float>> build_envs(const bcc_env_soa* s) {
    std::vector<Environment<float>> envs;
    envs.reserve(s->num_envs);
    size_t off[6] = {0, 0, 0, 0, 0, 0};
    auto cnt = [&](const uint32_t* c, int i) { return c ? c[i] : 0u; };
    for (int i = 0; i < s->num_envs; ++i) {
        Environment<float> e;
        e.num_spheres = cnt(s->num_spheres, i);
        e.num_capsules = cnt(s->num_capsules, i);
        e.num_z_aligned_capsules = cnt(s->num_z_capsules, i);
        e.num_cuboids = cnt(s->num_cuboids, i);
        e.num_z_aligned_cuboids = cnt(s->num_z_cuboids, i);
        e.num_cylinders = cnt(s->num_cylinders, i);
        e.spheres = e.num_spheres ? new Sphere<float>[e.num_spheres] : nullptr;
        e.capsules = e.num_capsules ? new Capsule<float>[e.num_capsules] : nullptr;
        e.z_aligned_capsules = e.num_z_aligned_capsules ? new Capsule<float>[e.num_z_aligned_capsules] : nullptr;
        e.cylinders = e.num_cylinders ? new Capsule<float>[e.num_cylinders] : nullptr;
        e.cuboids = e.num_cuboids ? new Cuboid<float>[e.num_cuboids] : nullptr;
        e.z_aligned_cuboids = e.num_z_aligned_cuboids ? new Cuboid<float>[e.num_z_aligned_cuboids] : nullptr;
        for (unsigned j = 0; j < e.num_spheres; ++j) {
            const float* r = s->spheres + 4 * (off[0] + j);
            e.spheres[j] = Sphere<float>(r[0], r[1], r[2], r[3]);
        }
        auto caps = [&](Capsule<float>* dst, unsigned n, const float* base, size_t o) {
            for (unsigned j = 0; j < n; ++j) {
                const float* r = base + 8 * (o + j);
                dst[j] = Capsule<float>(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7]);
            }
        };
        auto cubs = [&](Cuboid<float>* dst, unsigned n, const float* base, size_t o) {
            for (unsigned j = 0; j < n; ++j) {
                const float* r = base + 15 * (o + j);
                dst[j] = Cuboid<float>(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9], r[10],
                                       r[11], r[12], r[13], r[14]);
            }
        };
        caps(e.capsules, e.num_capsules, s->capsules, off[1]);
        caps(e.z_aligned_capsules, e.num_z_aligned_capsules, s->z_capsules, off[2]);
        cubs(e.cuboids, e.num_cuboids, s->cuboids, off[3]);
        cubs(e.z_aligned_cuboids, e.num_z_aligned_cuboids, s->z_cuboids, off[4]);
        caps(e.cylinders, e.num_cylinders, s->cylinders, off[5]);
        off[0] += e.num_spheres;
        off[1] += e.num_capsules;
        off[2] += e.num_z_aligned_capsules;
        off[3] += e.num_cuboids;
        off[4] += e.num_z_aligned_cuboids;
        off[5] += e.num_cylinders;
        envs.push_back(std::move(e));
    }
    return envs;
}

template <int DOF>
std::vector<std::array<std::array<float, DOF>, 2>> build_edges(const float* edges, int E) {
    std::vector<std::array<std::array<float, DOF>, 2>> v(E);
    for (int i = 0; i < E; ++i)
        for (int k = 0; k < 2; ++k)
            for (int j = 0; j < DOF; ++j) v[i][k][j] = edges[(size_t)i * 2 * DOF + k * DOF + j];
    return v;
}

}  // namespace

// Five-argument entry points of the reference's Fetch / Baxter check functions.
template <>
__device__ __forceinline__ bool ppln::collision::fkcc<ppln::robots::Fetch>(volatile float* q,
                                                                           ppln::collision::Environment<float>* env,
                                                                           int tid, int, int) {
    return ppln::collision::fkcc<ppln::robots::Fetch>(q, env, tid);
}
template <>
__device__ __forceinline__ bool ppln::collision::fkcc<ppln::robots::Baxter>(volatile float* q,
                                                                            ppln::collision::Environment<float>* env,
                                                                            int tid, int, int) {
    return ppln::collision::fkcc<ppln::robots::Baxter>(q, env, tid);
}
template void batch_cc::batch_cc<ppln::robots::Fetch>(
    std::vector<ppln::collision::Environment<float>>&,
    std::vector<std::array<typename ppln::robots::Fetch::Configuration, 2>>&, int, std::vector<bool>&);
template void batch_cc::batch_cc<ppln::robots::Baxter>(
    std::vector<ppln::collision::Environment<float>>&,
    std::vector<std::array<typename ppln::robots::Baxter::Configuration, 2>>&, int, std::vector<bool>&);

// Probe fkcc: records the configuration and reports "free" so every round runs.
template <>
__device__ __forceinline__ bool ppln::collision::fkcc<ProbeRobot>(volatile float* config,
                                                                  ppln::collision::Environment<float>*,
                                                                  int tid, int, int edge_idx) {
    const int i = atomicAdd(g_probe_count + edge_idx * 32 + tid, 1);
    if (i < kProbeRounds) {
        float* o = g_probe_out + (((size_t)edge_idx * 32 + tid) * kProbeRounds + i) * 7;
        for (int j = 0; j < 7; ++j) o[j] = config[j];
    }
    return true;
}

namespace {

template <class Robot>
int check_robot(const bcc_env_soa* envs, const float* edges, int E, int resolution, uint8_t* out, int quiet) {
    auto h_envs = build_envs(envs);
    auto h_edges = build_edges<Robot::dimension>(edges, E);
    std::vector<bool> results((size_t)E * envs->num_envs);
    {
        QuietStdout q(quiet != 0);
        batch_cc::batch_cc<Robot>(h_envs, h_edges, resolution, results);
    }
    for (size_t i = 0; i < results.size(); ++i) out[i] = results[i] ? 1 : 0;
    return (int)cudaGetLastError();
}

// Reference kernel on reference-placed environments; returns mean kernel ms
// over `iters` launches (after one warm-up), verdicts of the last launch.
template <class Robot>
int time_robot(const bcc_env_soa* envs, const float* edges, int E, int resolution, int iters, float* ms_out,
               uint8_t* out) {
    using EnvF = ppln::collision::Environment<float>;
    auto h_envs = build_envs(envs);
    const int N = envs->num_envs;
    const size_t edge_bytes = sizeof(float) * 2 * Robot::dimension * (size_t)E;
    std::vector<EnvF*> d_envs(N, nullptr);
    std::vector<void*> d_blobs;
    for (int i = 0; i < N; ++i) batch_cc::setup_environment_on_device(d_envs[i], h_envs[i], d_blobs);
    EnvF** d_envs_ptr = nullptr;
    float* d_edges = nullptr;
    bool* d_res = nullptr;
    cudaMalloc(&d_envs_ptr, sizeof(EnvF*) * N);
    cudaMemcpy(d_envs_ptr, d_envs.data(), sizeof(EnvF*) * N, cudaMemcpyHostToDevice);
    cudaMalloc(&d_edges, edge_bytes);
    cudaMemcpy(d_edges, edges, edge_bytes, cudaMemcpyHostToDevice);
    cudaMalloc(&d_res, (size_t)N * E);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const long long blocks = (long long)N * E;
    batch_cc::batch_cc_kernel<Robot><<<(unsigned)blocks, 32>>>(d_envs_ptr, d_edges, N, E, d_res, resolution);
    cudaEventRecord(a);
    for (int it = 0; it < iters; ++it)
        batch_cc::batch_cc_kernel<Robot><<<(unsigned)blocks, 32>>>(d_envs_ptr, d_edges, N, E, d_res, resolution);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    *ms_out = iters > 0 ? ms / iters : 0.0f;
    if (out) cudaMemcpy(out, d_res, (size_t)N * E, cudaMemcpyDeviceToHost);
    int err = (int)cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (int i = 0; i < N; ++i) batch_cc::cleanup_environment_on_device(d_envs[i], d_blobs[i]);
    cudaFree(d_envs_ptr);
    cudaFree(d_edges);
    cudaFree(d_res);
    return err;
}

}  // namespace

extern "C" {

// robot: BCC_ROBOT_PANDA / _FETCH / _BAXTER; -1 for an unknown robot.
int ref_check(int robot, const bcc_env_soa* envs, const float* edges, int E, int resolution, uint8_t* out,
              int quiet) {
    switch (robot) {
        case BCC_ROBOT_PANDA: return check_robot<ppln::robots::Panda>(envs, edges, E, resolution, out, quiet);
        case BCC_ROBOT_FETCH: return check_robot<ppln::robots::Fetch>(envs, edges, E, resolution, out, quiet);
        case BCC_ROBOT_BAXTER: return check_robot<ppln::robots::Baxter>(envs, edges, E, resolution, out, quiet);
        default: return -1;
    }
}

int ref_time(int robot, const bcc_env_soa* envs, const float* edges, int E, int resolution, int iters,
             float* ms_out, uint8_t* out) {
    switch (robot) {
        case BCC_ROBOT_PANDA:
            return time_robot<ppln::robots::Panda>(envs, edges, E, resolution, iters, ms_out, out);
        case BCC_ROBOT_FETCH:
            return time_robot<ppln::robots::Fetch>(envs, edges, E, resolution, iters, ms_out, out);
        case BCC_ROBOT_BAXTER:
            return time_robot<ppln::robots::Baxter>(envs, edges, E, resolution, iters, ms_out, out);
        default: return -1;
    }
}

// Configurations the reference kernel checks: out [E][32][16][7] (lane, round),
// counts [E][32] = rounds run per lane (== n; rounds beyond 16 not stored).
int ref_probe_samples(const float* edges, int E, int resolution, float* out, int* counts) {
    using EnvF = ppln::collision::Environment<float>;
    EnvF** d_envs_ptr = nullptr;
    float *d_edges = nullptr, *d_out = nullptr;
    int* d_cnt = nullptr;
    bool* d_res = nullptr;
    cudaMalloc(&d_envs_ptr, sizeof(EnvF*));
    cudaMemset(d_envs_ptr, 0, sizeof(EnvF*));
    cudaMalloc(&d_edges, sizeof(float) * 14 * (size_t)E);
    cudaMemcpy(d_edges, edges, sizeof(float) * 14 * (size_t)E, cudaMemcpyHostToDevice);
    const size_t n_out = (size_t)E * 32 * kProbeRounds * 7;
    cudaMalloc(&d_out, sizeof(float) * n_out);
    cudaMemset(d_out, 0, sizeof(float) * n_out);
    cudaMalloc(&d_cnt, sizeof(int) * 32 * (size_t)E);
    cudaMemset(d_cnt, 0, sizeof(int) * 32 * (size_t)E);
    cudaMalloc(&d_res, (size_t)E);
    cudaMemcpyToSymbol(g_probe_out, &d_out, sizeof(d_out));
    cudaMemcpyToSymbol(g_probe_count, &d_cnt, sizeof(d_cnt));
    batch_cc::batch_cc_kernel<ProbeRobot><<<E, 32>>>(d_envs_ptr, d_edges, 1, E, d_res, resolution);
    cudaDeviceSynchronize();
    cudaMemcpy(out, d_out, sizeof(float) * n_out, cudaMemcpyDeviceToHost);
    cudaMemcpy(counts, d_cnt, sizeof(int) * 32 * (size_t)E, cudaMemcpyDeviceToHost);
    int err = (int)cudaGetLastError();
    cudaFree(d_envs_ptr);
    cudaFree(d_edges);
    cudaFree(d_out);
    cudaFree(d_cnt);
    cudaFree(d_res);
    return err;
}

}  // extern "C"
