// loaders.hh -- environment loaders of the CLI driver.
//
// * MotionBenchMaker problem files (the reference driver's input,
//   scripts/batch_cc_mbm.cpp:19-123): problem families in key order, invalid
//   problems skipped; spheres as spheres, boxes as cuboids (centre, Euler XYZ,
//   half-extents); cylinders as capsules of the given radius and length --
//   except in the "box" family, where each cylinder becomes a cuboid with
//   half-extents (r, r, r/2).
// * scene files (scripts/batch_cc.cpp:82-278): OBJECT primitives shared by all
//   environments, OBSTACLEk_ / TARGET_ lines giving environment i its i-th
//   sample; BOX dims are full extents, orientations quaternions (x y z w).
#pragma once

#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "json_lite.hh"
#include "src/collision/environment.hh"
#include "src/collision/factory.hh"

namespace bcc_loaders {

using ppln::collision::Capsule;
using ppln::collision::Cuboid;
using ppln::collision::Environment;
using ppln::collision::Sphere;
namespace factory = ppln::collision::factory;

inline std::string read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

inline std::array<float, 3> vec3(const bcc_json::Value& v) { return {v[0].f(), v[1].f(), v[2].f()}; }

template <class T>
inline void fill(T*& dst, unsigned int& n, const std::vector<T>& src) {
    n = (unsigned int)src.size();
    dst = src.empty() ? nullptr : new T[src.size()];
    for (size_t i = 0; i < src.size(); ++i) dst[i] = src[i];
}

inline Environment<float> problem_to_env(const bcc_json::Value& p, const std::string& family) {
    std::vector<Sphere<float>> spheres;
    std::vector<Capsule<float>> capsules;
    std::vector<Cuboid<float>> cuboids;
    for (const auto& o : p["sphere"].arr) {
        Sphere<float> s(o["position"][0].f(), o["position"][1].f(), o["position"][2].f(), o["radius"].f());
        s.name = o["name"].str;
        spheres.push_back(s);
    }
    for (const auto& o : p["cylinder"].arr) {
        const float r = o["radius"].f();
        if (family == "box") {
            auto c = factory::cuboid::array(vec3(o["position"]), vec3(o["orientation_euler_xyz"]), {r, r, r / 2.0f});
            c.name = o["name"].str;
            cuboids.push_back(c);
        } else {
            auto c = factory::cylinder::center::array(vec3(o["position"]), vec3(o["orientation_euler_xyz"]), r,
                                                      o["length"].f());
            c.name = o["name"].str;
            capsules.push_back(c);
        }
    }
    for (const auto& o : p["box"].arr) {
        auto c = factory::cuboid::array(vec3(o["position"]), vec3(o["orientation_euler_xyz"]), vec3(o["half_extents"]));
        c.name = o["name"].str;
        cuboids.push_back(c);
    }
    Environment<float> env;
    fill(env.spheres, env.num_spheres, spheres);
    fill(env.capsules, env.num_capsules, capsules);
    fill(env.cuboids, env.num_cuboids, cuboids);
    return env;
}

inline std::vector<Environment<float>> load_mbm(const std::string& path, int num_envs) {
    const bcc_json::Value root = bcc_json::parse(read_file(path));
    std::vector<Environment<float>> envs;
    for (const auto& fam : root["problems"].obj) {
        for (const auto& p : fam.second.arr) {
            if ((int)envs.size() >= num_envs) return envs;
            if (!p["valid"].b) continue;
            envs.push_back(problem_to_env(p, fam.first));
        }
    }
    return envs;
}

inline std::array<float, 3> quat_to_euler(float x, float y, float z, float w) {
    const float roll = std::atan2(2.0f * (w * x + y * z), 1.0f - 2.0f * (x * x + y * y));
    const float pitch = std::asin(std::max(-1.0f, std::min(1.0f, 2.0f * (w * y - z * x))));
    const float yaw = std::atan2(2.0f * (w * z + x * y), 1.0f - 2.0f * (y * y + z * z));
    return {roll, pitch, yaw};
}

inline std::vector<Environment<float>> load_scene(const std::string& path, int num_envs) {
    std::istringstream in(read_file(path));
    std::vector<Sphere<float>> obj_s;
    std::vector<Cuboid<float>> obj_b;
    std::vector<Capsule<float>> obj_c;
    // per sampled group (OBSTACLEk_ / TARGET_, in name order): samples in file order
    std::map<std::string, std::vector<Sphere<float>>> grp_s;
    std::map<std::string, std::vector<Cuboid<float>>> grp_b;
    std::map<std::string, std::vector<Capsule<float>>> grp_c;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string cat, type;
        if (!(ls >> cat >> type)) continue;
        const bool sampled = !cat.empty() && cat.back() == '_';
        const bool object = cat.find("OBJECT") != std::string::npos;
        if (!sampled && !object) continue;  // the mean pose of a sampled group
        const std::string group = sampled ? cat.substr(0, cat.size() - 1) : cat;
        if (type == "BOX") {
            float x, y, z, qx, qy, qz, qw, dx, dy, dz;
            ls >> x >> y >> z >> qx >> qy >> qz >> qw >> dx >> dy >> dz;
            auto c = factory::cuboid::array({x, y, z}, quat_to_euler(qx, qy, qz, qw), {dx / 2, dy / 2, dz / 2});
            (object ? obj_b : grp_b[group]).push_back(c);
        } else if (type == "SPHERE") {
            float x, y, z, r;
            ls >> x >> y >> z >> r;
            (object ? obj_s : grp_s[group]).push_back(Sphere<float>(x, y, z, r));
        } else if (type == "CYLINDER") {
            float x, y, z, qx, qy, qz, qw, h, r;
            ls >> x >> y >> z >> qx >> qy >> qz >> qw >> h >> r;
            auto c = factory::cylinder::center::array({x, y, z}, quat_to_euler(qx, qy, qz, qw), r, h);
            (object ? obj_c : grp_c[group]).push_back(c);
        }
    }
    std::vector<Environment<float>> envs;
    for (int i = 0; i < num_envs; ++i) {
        std::vector<Sphere<float>> s = obj_s;
        std::vector<Cuboid<float>> b = obj_b;
        std::vector<Capsule<float>> c = obj_c;
        // obstacle groups before the target group (OBSTACLE* < TARGET in name order)
        for (auto& g : grp_b)
            if (i < (int)g.second.size()) b.push_back(g.second[i]);
        for (auto& g : grp_s)
            if (i < (int)g.second.size()) s.push_back(g.second[i]);
        for (auto& g : grp_c)
            if (i < (int)g.second.size()) c.push_back(g.second[i]);
        Environment<float> env;
        fill(env.spheres, env.num_spheres, s);
        fill(env.cuboids, env.num_cuboids, b);
        fill(env.capsules, env.num_capsules, c);
        envs.push_back(std::move(env));
    }
    return envs;
}

}  // namespace bcc_loaders
