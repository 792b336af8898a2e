// A collision environment: arrays of primitives by kind (drop-in for the
// reference header src/collision/environment.hh, same members).  An
// environment that owns its arrays (owns_memory, the default) delete[]s them.
#pragma once

#include "shapes.hh"

namespace ppln::collision {

template <typename T>
struct Environment {
    Sphere<T>* spheres = nullptr;
    unsigned int num_spheres = 0;
    Capsule<T>* capsules = nullptr;
    unsigned int num_capsules = 0;
    Capsule<T>* z_aligned_capsules = nullptr;
    unsigned int num_z_aligned_capsules = 0;
    Cylinder<T>* cylinders = nullptr;
    unsigned int num_cylinders = 0;
    Cuboid<T>* cuboids = nullptr;
    unsigned int num_cuboids = 0;
    Cuboid<T>* z_aligned_cuboids = nullptr;
    unsigned int num_z_aligned_cuboids = 0;
    bool owns_memory = true;

    Environment() = default;
    Environment(const Environment&) = delete;
    Environment& operator=(const Environment&) = delete;
    Environment(Environment&& o) noexcept { take(o); }
    Environment& operator=(Environment&& o) noexcept {
        if (this != &o) {
            release();
            take(o);
        }
        return *this;
    }
    ~Environment() { release(); }

  private:
    void take(Environment& o) {
        spheres = o.spheres, num_spheres = o.num_spheres;
        capsules = o.capsules, num_capsules = o.num_capsules;
        z_aligned_capsules = o.z_aligned_capsules, num_z_aligned_capsules = o.num_z_aligned_capsules;
        cylinders = o.cylinders, num_cylinders = o.num_cylinders;
        cuboids = o.cuboids, num_cuboids = o.num_cuboids;
        z_aligned_cuboids = o.z_aligned_cuboids, num_z_aligned_cuboids = o.num_z_aligned_cuboids;
        owns_memory = o.owns_memory;
        o.spheres = nullptr, o.capsules = nullptr, o.z_aligned_capsules = nullptr;
        o.cylinders = nullptr, o.cuboids = nullptr, o.z_aligned_cuboids = nullptr;
        o.owns_memory = false;
    }
    void release() {
        if (!owns_memory) return;
        delete[] spheres;
        delete[] capsules;
        delete[] z_aligned_capsules;
        delete[] cylinders;
        delete[] cuboids;
        delete[] z_aligned_cuboids;
        spheres = nullptr;
        capsules = z_aligned_capsules = cylinders = nullptr;
        cuboids = z_aligned_cuboids = nullptr;
    }
};

}  // namespace ppln::collision
