// Drop-in for the reference entry point src/batch_cc.hh:
//
//   template <typename Robot>
//   void batch_cc::batch_cc(std::vector<ppln::collision::Environment<float>>& h_envs,
//                           std::vector<std::array<typename Robot::Configuration, 2>>& edges,
//                           int resolution, std::vector<bool>& results);
//
// Header-only adapter over the C ABI (include/bcc.h, link libbcc.so): the
// environments are repacked member by member into the ABI's
// structure-of-arrays form, uploaded into a per-device context kept for the
// life of the process, and checked on the GPU.  results must be pre-sized to
// num_envs * num_edges (as in the reference) and receives
// results[edge * num_envs + env] = true when the edge collides in that env.
// Errors throw std::runtime_error.  Like the reference it prints its setup,
// kernel and throughput lines to stdout; set BCC_QUIET=1 to silence them.
#pragma once

#include <array>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../bcc.h"
#include "Robots.hh"
#include "collision/environment.hh"

namespace batch_cc {

namespace detail {

inline bcc_ctx* context() {
    static bcc_ctx* ctx = [] {
        bcc_ctx* c = nullptr;
        if (bcc_create(&c, 0) != BCC_OK) throw std::runtime_error("bcc_create failed (no CUDA device?)");
        return c;
    }();
    return ctx;
}

template <typename Robot>
inline bcc_robot robot_id() {
    const std::string n = Robot::name;
    if (n == "panda") return BCC_ROBOT_PANDA;
    if (n == "fetch") return BCC_ROBOT_FETCH;
    if (n == "baxter") return BCC_ROBOT_BAXTER;
    throw std::runtime_error("robot " + n + " is not supported");
}

inline bool quiet() {
    const char* q = std::getenv("BCC_QUIET");
    return q && q[0] == '1';
}

struct Packed {
    std::vector<uint32_t> ns, nc, nzc, nb, nzb, ncy;
    std::vector<float> s, c, zc, b, zb, cy;
};

inline void pack_capsule(std::vector<float>& dst, const ppln::collision::Capsule<float>& x) {
    dst.insert(dst.end(), {x.x1, x.y1, x.z1, x.xv, x.yv, x.zv, x.r, x.rdv});
}

inline void pack_cuboid(std::vector<float>& dst, const ppln::collision::Cuboid<float>& x) {
    dst.insert(dst.end(), {x.x, x.y, x.z, x.axis_1_x, x.axis_1_y, x.axis_1_z, x.axis_2_x, x.axis_2_y, x.axis_2_z,
                           x.axis_3_x, x.axis_3_y, x.axis_3_z, x.axis_1_r, x.axis_2_r, x.axis_3_r});
}

inline Packed pack(const std::vector<ppln::collision::Environment<float>>& envs) {
    Packed p;
    for (const auto& e : envs) {
        // ensure_ptr_count_consistent (reference src/batch_cc.cu:45-56)
        if ((e.num_spheres && !e.spheres) || (e.num_capsules && !e.capsules) ||
            (e.num_z_aligned_capsules && !e.z_aligned_capsules) || (e.num_cylinders && !e.cylinders) ||
            (e.num_cuboids && !e.cuboids) || (e.num_z_aligned_cuboids && !e.z_aligned_cuboids))
            throw std::runtime_error("Host environment has positive counts with null pointers.");
        p.ns.push_back(e.num_spheres);
        for (unsigned i = 0; i < e.num_spheres; ++i) {
            const auto& x = e.spheres[i];
            p.s.insert(p.s.end(), {x.x, x.y, x.z, x.r});
        }
        p.nc.push_back(e.num_capsules);
        for (unsigned i = 0; i < e.num_capsules; ++i) pack_capsule(p.c, e.capsules[i]);
        p.nzc.push_back(e.num_z_aligned_capsules);
        for (unsigned i = 0; i < e.num_z_aligned_capsules; ++i) pack_capsule(p.zc, e.z_aligned_capsules[i]);
        p.nb.push_back(e.num_cuboids);
        for (unsigned i = 0; i < e.num_cuboids; ++i) pack_cuboid(p.b, e.cuboids[i]);
        p.nzb.push_back(e.num_z_aligned_cuboids);
        for (unsigned i = 0; i < e.num_z_aligned_cuboids; ++i) pack_cuboid(p.zb, e.z_aligned_cuboids[i]);
        p.ncy.push_back(e.num_cylinders);
        for (unsigned i = 0; i < e.num_cylinders; ++i) pack_capsule(p.cy, e.cylinders[i]);
    }
    return p;
}

template <class T>
inline const T* ptr(const std::vector<T>& v) {
    return v.empty() ? nullptr : v.data();
}

}  // namespace detail

template <typename Robot>
void batch_cc(std::vector<ppln::collision::Environment<float>>& h_envs,
              std::vector<std::array<typename Robot::Configuration, 2>>& edges, int resolution,
              std::vector<bool>& results) {
    using clock = std::chrono::steady_clock;
    const bool q = detail::quiet();
    const auto t_setup = clock::now();
    bcc_ctx* ctx = detail::context();
    const detail::Packed p = detail::pack(h_envs);
    bcc_env_soa soa{(int32_t)h_envs.size(), detail::ptr(p.ns), detail::ptr(p.nc), detail::ptr(p.nzc),
                    detail::ptr(p.nb), detail::ptr(p.nzb), detail::ptr(p.ncy), detail::ptr(p.s), detail::ptr(p.c),
                    detail::ptr(p.zc), detail::ptr(p.b), detail::ptr(p.zb), detail::ptr(p.cy)};
    if (bcc_upload_envs(ctx, &soa) != BCC_OK) throw std::runtime_error(bcc_last_error(ctx));
    const size_t N = h_envs.size(), E = edges.size();
    if (results.size() < N * E) throw std::runtime_error("results must be pre-sized to num_envs * num_edges");
    std::vector<float> flat(E * 2 * Robot::dimension);
    for (size_t i = 0; i < E; ++i)
        for (int k = 0; k < 2; ++k)
            for (int j = 0; j < Robot::dimension; ++j) flat[(i * 2 + k) * Robot::dimension + j] = edges[i][k][j];
    std::vector<uint8_t> out(N * E);
    const double setup_s = std::chrono::duration<double>(clock::now() - t_setup).count();
    if (!q) std::cout << "Setup time: " << setup_s << " s" << std::endl;
    const auto t_kernel = clock::now();
    if (N * E > 0 &&
        bcc_check(ctx, detail::robot_id<Robot>(), flat.data(), (int32_t)E, resolution, out.data(), nullptr) != BCC_OK)
        throw std::runtime_error(bcc_last_error(ctx));
    const auto kernel_ns = std::chrono::duration_cast<std::chrono::nanoseconds>(clock::now() - t_kernel).count();
    if (!q) {
        std::cout << "Kernel time: " << kernel_ns << " ns" << std::endl;
        std::cout << "Edges checked: " << N * E << std::endl;
        std::cout << "Throughput: " << (double)(N * E) / (kernel_ns / 1e9) << " edges/s" << std::endl;
    }
    for (size_t i = 0; i < N * E; ++i) results[i] = out[i] != 0;
}

}  // namespace batch_cc
