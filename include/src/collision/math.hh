// Small vector helpers of the collision data model (drop-in for the reference
// header src/collision/math.hh: same names and argument order).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>

namespace ppln::collision {

using Point = std::array<float, 3>;

template <typename T>
inline constexpr T dot_2(const T& ax, const T& ay, const T& bx, const T& by) {
    return ax * bx + ay * by;
}

template <typename T>
inline constexpr T dot_3(const T& ax, const T& ay, const T& az, const T& bx, const T& by, const T& bz) {
    return ax * bx + ay * by + az * bz;
}

template <typename T>
inline constexpr T sql2_3(const T& ax, const T& ay, const T& az, const T& bx, const T& by, const T& bz) {
    const T dx = ax - bx, dy = ay - by, dz = az - bz;
    return dx * dx + dy * dy + dz * dz;
}

inline constexpr float clamp(const float& v, const float& lo, const float& hi) { return std::max(std::min(v, hi), lo); }

}  // namespace ppln::collision
