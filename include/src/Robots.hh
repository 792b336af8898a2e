// Robot descriptions (drop-in for the reference header src/Robots.hh): name,
// degrees of freedom, configuration type and the joint-limit scale
// q = u * s_m + s_a that maps a unit-cube sample into the limits.  The limit
// values are the reference's (src/Robots.hh:17-41 Panda, :72-98 Fetch,
// :128-166 Baxter).
#pragma once

#include <array>
#include <cstddef>
#include <iostream>

#if defined(__CUDACC__)
#define BCC_HD __host__ __device__
#else
#define BCC_HD
#endif

namespace ppln::robots {

template <class Derived, int Dof>
struct RobotBase {
    static constexpr auto dimension = Dof;
    using Configuration = std::array<float, Dof>;

    static void print_robot_config(Configuration& cfg) {
        for (int i = 0; i < Dof; ++i) std::cout << cfg[i] << ' ';
        std::cout << '\n';
    }
    BCC_HD static void scale_cfg(float* q) {
        for (int i = 0; i < Dof; ++i) q[i] = q[i] * Derived::get_s_m(i) + Derived::get_s_a(i);
    }
};

struct Panda : RobotBase<Panda, 7> {
    static constexpr auto name = "panda";
    BCC_HD static constexpr float get_s_m(int i) {
        constexpr float v[] = {5.9342f, 3.6652f, 5.9342f, 3.2289f, 5.9342f, 3.9095999999999997f, 5.9342f};
        return v[i];
    }
    BCC_HD static constexpr float get_s_a(int i) {
        constexpr float v[] = {-2.9671f, -1.8326f, -2.9671f, -3.1416f, -2.9671f, -0.0873f, -2.9671f};
        return v[i];
    }
};

struct Fetch : RobotBase<Fetch, 8> {
    static constexpr auto name = "fetch";
    BCC_HD static constexpr float get_s_m(int i) {
        constexpr float v[] = {0.38615f, 3.2112f, 2.739f, 6.28318f, 4.502f, 6.28318f, 4.32f, 6.28318f};
        return v[i];
    }
    BCC_HD static constexpr float get_s_a(int i) {
        constexpr float v[] = {0.0f, -1.6056f, -1.221f, -3.14159f, -2.251f, -3.14159f, -2.16f, -3.14159f};
        return v[i];
    }
};

struct Baxter : RobotBase<Baxter, 14> {
    static constexpr auto name = "baxter";
    BCC_HD static constexpr float get_s_m(int i) {
        constexpr float v[] = {3.40335987756f, 3.194f, 6.10835987756f, 2.6679999999999997f, 6.118f, 3.66479632679f, 6.118f,
                               3.40335987756f, 3.194f, 6.10835987756f, 2.6679999999999997f, 6.118f, 3.66479632679f, 6.118f};
        return v[i];
    }
    BCC_HD static constexpr float get_s_a(int i) {
        constexpr float v[] = {-1.70167993878f, -2.147f, -3.05417993878f, -0.05f, -3.059f, -1.57079632679f, -3.059f,
                               -1.70167993878f, -2.147f, -3.05417993878f, -0.05f, -3.059f, -1.57079632679f, -3.059f};
        return v[i];
    }
};

}  // namespace ppln::robots
