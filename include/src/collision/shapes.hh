// Collision primitives (drop-in for the reference header
// src/collision/shapes.hh).  Member names, member order and constructor
// argument order are those of the reference so that callers can fill them
// member by member; every shape carries a name and a min_distance (distance
// from the origin, computed at construction).
#pragma once

#include <cmath>
#include <string>

#include "math.hh"

namespace ppln::collision {

template <typename T>
struct Shape {
    std::string name;
    T min_distance{};
    Shape() = default;
    template <typename U>
    explicit Shape(const Shape<U>& o) : name(o.name), min_distance(o.min_distance) {}
};

// Oriented box: centre, three unit axes, half-extents along them.
template <typename T>
struct Cuboid : public Shape<T> {
    T x, y, z;
    T axis_1_x, axis_1_y, axis_1_z;
    T axis_2_x, axis_2_y, axis_2_z;
    T axis_3_x, axis_3_y, axis_3_z;
    T axis_1_r, axis_2_r, axis_3_r;

    Cuboid() = default;
    explicit Cuboid(T x_, T y_, T z_, T a1x, T a1y, T a1z, T a2x, T a2y, T a2z, T a3x, T a3y, T a3z, T r1, T r2, T r3)
        : x(x_), y(y_), z(z_), axis_1_x(a1x), axis_1_y(a1y), axis_1_z(a1z), axis_2_x(a2x), axis_2_y(a2y),
          axis_2_z(a2z), axis_3_x(a3x), axis_3_y(a3y), axis_3_z(a3z), axis_1_r(r1), axis_2_r(r2), axis_3_r(r3) {
        // closest point of the box to the origin
        const T p1 = clamp(dot_3(-x, -y, -z, a1x, a1y, a1z), -r1, r1);
        const T p2 = clamp(dot_3(-x, -y, -z, a2x, a2y, a2z), -r2, r2);
        const T p3 = clamp(dot_3(-x, -y, -z, a3x, a3y, a3z), -r3, r3);
        const T cx = x + a1x * p1 + a2x * p2 + a3x * p3;
        const T cy = y + a1y * p1 + a2y * p2 + a3y * p3;
        const T cz = z + a1z * p1 + a2z * p2 + a3z * p3;
        this->min_distance = std::sqrt(cx * cx + cy * cy + cz * cz);
    }
};

// Segment p1 -> p1 + v swept by a sphere of radius r; rdv = 1 / |v|^2.
template <typename T>
struct Cylinder : public Shape<T> {
    T x1, y1, z1;
    T xv, yv, zv;
    T r;
    T rdv;

    Cylinder() = default;
    explicit Cylinder(T x1_, T y1_, T z1_, T xv_, T yv_, T zv_, T r_, T rdv_)
        : x1(x1_), y1(y1_), z1(z1_), xv(xv_), yv(yv_), zv(zv_), r(r_), rdv(rdv_) {
        const T t = clamp(dot_3(-x1, -y1, -z1, xv, yv, zv) * rdv, T(0), T(1));
        const T px = x1 + xv * t, py = y1 + yv * t, pz = z1 + zv * t;
        const T d = std::sqrt(px * px + py * py + pz * pz);
        const T along = clamp(d, T(0), r);
        const T s = d > T(0) ? (d - along) / d : T(0);
        this->min_distance = std::sqrt((px * s) * (px * s) + (py * s) * (py * s) + (pz * s) * (pz * s));
    }
    constexpr T x2() const { return x1 + xv; }
    constexpr T y2() const { return y1 + yv; }
    constexpr T z2() const { return z1 + zv; }
};

template <typename T>
using Capsule = Cylinder<T>;

template <typename T>
struct Sphere : public Shape<T> {
    T x, y, z, r;
    Sphere() = default;
    explicit Sphere(T x_, T y_, T z_, T r_) : x(x_), y(y_), z(z_), r(r_) {
        this->min_distance = std::sqrt(x * x + y * y + z * z) - r;
    }
};

}  // namespace ppln::collision
