// batch_cc -- command-line driver, drop-in for the reference drivers:
//
//     batch_cc <robot_name> <num_environments> <num_edges> [problems.json | scene.txt]
//         (scripts/batch_cc_mbm.cpp:181-207) environments from the
//         MotionBenchMaker problem file scripts/<robot>_problems.json (or the
//         given file; a .txt file is read as a scene file); edges are
//         consecutive Halton samples scaled into the joint limits;
//     batch_cc <robot_name> <graph.dot> <scene.txt>
//         (scripts/batch_cc.cpp:331-425) the edges of a roadmap graph whose
//         vertices carry `states`, checked in all 200 scene environments.
//
// Resolution 32.  Prints the checker's timing lines and one line
// "Edge i: v v v ..." per edge (v = 1 when the edge collides in environment j).
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "dot.hh"
#include "loaders.hh"
#include "src/Robots.hh"
#include "src/batch_cc.hh"
#include "src/random/halton.hh"

// Inputs as checked, for tests: int32 num_envs, num_edges, dof; per env the
// sphere, capsule and cuboid counts (int32 x 3); then the records of all envs
// (spheres 4, capsules 8, cuboids 15 floats, env by env); then the edges.
template <typename Robot>
void dump_inputs(const char* path, const std::vector<ppln::collision::Environment<float>>& envs,
                 const std::vector<std::array<typename Robot::Configuration, 2>>& edges) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return;
    const int32_t hdr[3] = {(int32_t)envs.size(), (int32_t)edges.size(), Robot::dimension};
    std::fwrite(hdr, sizeof(hdr), 1, f);
    for (const auto& e : envs) {
        const int32_t c[3] = {(int32_t)e.num_spheres, (int32_t)e.num_capsules, (int32_t)e.num_cuboids};
        std::fwrite(c, sizeof(c), 1, f);
    }
    for (const auto& e : envs) {
        for (unsigned i = 0; i < e.num_spheres; ++i) {
            const auto& x = e.spheres[i];
            const float v[4] = {x.x, x.y, x.z, x.r};
            std::fwrite(v, sizeof(v), 1, f);
        }
        for (unsigned i = 0; i < e.num_capsules; ++i) {
            const auto& x = e.capsules[i];
            const float v[8] = {x.x1, x.y1, x.z1, x.xv, x.yv, x.zv, x.r, x.rdv};
            std::fwrite(v, sizeof(v), 1, f);
        }
        for (unsigned i = 0; i < e.num_cuboids; ++i) {
            const auto& x = e.cuboids[i];
            const float v[15] = {x.x, x.y, x.z, x.axis_1_x, x.axis_1_y, x.axis_1_z, x.axis_2_x, x.axis_2_y,
                                 x.axis_2_z, x.axis_3_x, x.axis_3_y, x.axis_3_z, x.axis_1_r, x.axis_2_r, x.axis_3_r};
            std::fwrite(v, sizeof(v), 1, f);
        }
    }
    for (const auto& ed : edges) std::fwrite(ed.data(), sizeof(ed), 1, f);
    std::fclose(f);
}

template <typename Robot>
int run(int num_envs, int num_edges, const std::string& path) {
    const bool scene = path.size() > 4 && path.substr(path.size() - 4) == ".txt";
    std::vector<ppln::collision::Environment<float>> envs =
        scene ? bcc_loaders::load_scene(path, num_envs) : bcc_loaders::load_mbm(path, num_envs);
    rng::Halton<Robot::dimension> halton;
    std::vector<std::array<typename Robot::Configuration, 2>> edges(num_edges);
    for (int i = 0; i < num_edges; ++i) {
        auto a = halton.next();
        auto b = halton.next();
        Robot::scale_cfg(a.data());
        Robot::scale_cfg(b.data());
        for (int j = 0; j < Robot::dimension; ++j) {
            edges[i][0][j] = a[j];
            edges[i][1][j] = b[j];
        }
    }
    if (const char* dump = std::getenv("BCC_DUMP_INPUTS")) dump_inputs<Robot>(dump, envs, edges);
    std::vector<bool> results((size_t)num_edges * envs.size());
    batch_cc::batch_cc<Robot>(envs, edges, 32, results);
    for (int i = 0; i < num_edges; ++i) {
        std::cout << "Edge " << i << ": ";
        for (size_t j = 0; j < envs.size(); ++j) std::cout << results[(size_t)i * envs.size() + j] << " ";
        std::cout << "\n";
    }
    return 0;
}

// Environments a scene file defines (MAX_WORLD_SAMPLES_EVAL, scripts/batch_cc.cpp:25).
constexpr int kSceneEnvs = 200;

template <typename Robot>
int run_graph(const std::string& graph_path, const std::string& scene_path) {
    std::vector<ppln::collision::Environment<float>> envs = bcc_loaders::load_scene(scene_path, kSceneEnvs);
    const bcc_dot::Graph g = bcc_dot::parse(bcc_loaders::read_file(graph_path));
    std::vector<std::array<typename Robot::Configuration, 2>> edges;
    edges.reserve(g.edges.size());
    for (const auto& e : g.edges) {
        const auto& a = g.states[e.first];
        const auto& b = g.states[e.second];
        if ((int)a.size() < Robot::dimension || (int)b.size() < Robot::dimension)
            throw std::runtime_error("graph vertex with fewer states than the robot's joints");
        std::array<typename Robot::Configuration, 2> edge;
        for (int i = 0; i < Robot::dimension; ++i) {
            edge[0][i] = (float)a[i];
            edge[1][i] = (float)b[i];
        }
        edges.push_back(edge);
    }
    std::cout << "Number of edges: " << edges.size() << "\n";
    std::cout << "Number of environments: " << envs.size() << "\n";
    if (const char* dump = std::getenv("BCC_DUMP_INPUTS")) dump_inputs<Robot>(dump, envs, edges);
    std::vector<bool> results(edges.size() * envs.size());
    batch_cc::batch_cc<Robot>(envs, edges, 32, results);
    for (size_t i = 0; i < edges.size(); ++i) {
        std::cout << "Edge " << i << ": ";
        for (size_t j = 0; j < envs.size(); ++j) std::cout << results[i * envs.size() + j] << " ";
        std::cout << "\n";
    }
    for (size_t i = 0; i < envs.size(); ++i)
        std::cout << "Environment " << i << ": " << envs[i].num_spheres << " spheres, " << envs[i].num_cuboids
                  << " cuboids, " << envs[i].num_capsules << " capsules\n\n";
    return 0;
}

inline bool ends_with(const std::string& s, const std::string& t) {
    return s.size() >= t.size() && s.compare(s.size() - t.size(), t.size(), t) == 0;
}

int main(int argc, char** argv) {
    if (argc == 4 && ends_with(argv[2], ".dot")) {  // roadmap graph mode
        const std::string robot = argv[1];
        try {
            if (robot == "panda") return run_graph<ppln::robots::Panda>(argv[2], argv[3]);
            if (robot == "fetch") return run_graph<ppln::robots::Fetch>(argv[2], argv[3]);
            if (robot == "baxter") return run_graph<ppln::robots::Baxter>(argv[2], argv[3]);
        } catch (const std::exception& e) {
            std::cerr << "batch_cc: " << e.what() << "\n";
            return 2;
        }
        std::cout << "Unknown robot name: " << robot << "\n";
        return -1;
    }
    if (argc != 4 && argc != 5) {
        std::cout << "Usage: ./batch_cc <robot_name> <num_environments> <num_edges>\n"
                     "       ./batch_cc <robot_name> <graph.dot> <scene.txt>\n";
        return 1;
    }
    const std::string robot = argv[1];
    const int num_envs = std::stoi(argv[2]);
    const int num_edges = std::stoi(argv[3]);
    const std::string path = argc == 5 ? argv[4] : "scripts/" + robot + "_problems.json";
    try {
        if (robot == "panda") return run<ppln::robots::Panda>(num_envs, num_edges, path);
        if (robot == "fetch") return run<ppln::robots::Fetch>(num_envs, num_edges, path);
        if (robot == "baxter") return run<ppln::robots::Baxter>(num_envs, num_edges, path);
    } catch (const std::exception& e) {
        std::cerr << "batch_cc: " << e.what() << "\n";
        return 2;
    }
    std::cout << "Unknown robot name: " << robot << "\n";
    return -1;
}
