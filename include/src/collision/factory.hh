// Shape builders (drop-in for the array/flat overloads of the reference header
// src/collision/factory.hh, without its Eigen dependency).  Orientation is
// Euler XYZ (rho, theta, phi) applied as R = Rz(phi) * Ry(theta) * Rx(rho); a
// cylinder / capsule of `length` about `center` spans center +- R (0, 0, length/2).
#pragma once

#include <array>
#include <cmath>

#include "shapes.hh"

namespace ppln::collision::factory {

using ConstArrayRef = const std::array<float, 3>&;

namespace detail {
inline std::array<float, 9> euler_xyz(float rho, float theta, float phi) {
    const float cr = std::cos(rho), sr = std::sin(rho), ct = std::cos(theta), st = std::sin(theta);
    const float cp = std::cos(phi), sp = std::sin(phi);
    // row-major Rz(phi) * Ry(theta) * Rx(rho)
    return {cp * ct, cp * st * sr - sp * cr, cp * st * cr + sp * sr,
            sp * ct, sp * st * sr + cp * cr, sp * st * cr - cp * sr,
            -st,     ct * sr,                ct * cr};
}
}  // namespace detail

namespace cuboid {
inline Cuboid<float> flat(float cx, float cy, float cz, float rho, float theta, float phi, float hx, float hy,
                          float hz) {
    const auto R = detail::euler_xyz(rho, theta, phi);
    // axes are the columns of R
    return Cuboid<float>(cx, cy, cz, R[0], R[3], R[6], R[1], R[4], R[7], R[2], R[5], R[8], hx, hy, hz);
}
inline Cuboid<float> array(ConstArrayRef c, ConstArrayRef euler, ConstArrayRef half) {
    return flat(c[0], c[1], c[2], euler[0], euler[1], euler[2], half[0], half[1], half[2]);
}
}  // namespace cuboid

namespace cylinder {
namespace endpoints {
inline Cylinder<float> flat(float x1, float y1, float z1, float x2, float y2, float z2, float radius) {
    const float vx = x2 - x1, vy = y2 - y1, vz = z2 - z1;
    const float dot = vx * vx + vy * vy + vz * vz;
    return Cylinder<float>(x1, y1, z1, vx, vy, vz, radius, static_cast<float>(1.0 / dot));
}
inline Cylinder<float> array(ConstArrayRef a, ConstArrayRef b, float radius) {
    return flat(a[0], a[1], a[2], b[0], b[1], b[2], radius);
}
}  // namespace endpoints
namespace center {
inline Cylinder<float> flat(float cx, float cy, float cz, float rho, float theta, float phi, float radius,
                            float length) {
    const auto R = detail::euler_xyz(rho, theta, phi);
    const float h = length / 2;
    const float ax = R[2] * h, ay = R[5] * h, az = R[8] * h;
    return endpoints::flat(cx + ax, cy + ay, cz + az, cx - ax, cy - ay, cz - az, radius);
}
inline Cylinder<float> array(ConstArrayRef c, ConstArrayRef euler, float radius, float length) {
    return flat(c[0], c[1], c[2], euler[0], euler[1], euler[2], radius, length);
}
}  // namespace center
}  // namespace cylinder

namespace capsule {
namespace endpoints = cylinder::endpoints;
namespace center = cylinder::center;
}  // namespace capsule

namespace sphere {
inline Sphere<float> flat(float cx, float cy, float cz, float r) { return Sphere<float>(cx, cy, cz, r); }
inline Sphere<float> array(ConstArrayRef c, float r) { return flat(c[0], c[1], c[2], r); }
}  // namespace sphere

}  // namespace ppln::collision::factory

using namespace ppln;
