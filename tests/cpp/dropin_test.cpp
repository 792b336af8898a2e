// Host-only checks of the drop-in headers (no GPU): prints values the Python
// test compares with independent computations.
#include <cmath>
#include <cstdio>
#include <string>

#include "loaders.hh"
#include "src/Robots.hh"
#include "src/random/halton.hh"

int main(int argc, char** argv) {
    const std::string mode = argv[1];
    if (mode == "halton") {
        rng::Halton<7> h;
        for (int i = 0; i < 2000; ++i) {
            auto v = h.next();
            for (float x : v) std::printf("%.9g ", x);
            std::printf("\n");
        }
    } else if (mode == "scale") {
        float q[7] = {0, 0.25f, 0.5f, 0.75f, 1, 0.1f, 0.9f};
        ppln::robots::Panda::scale_cfg(q);
        for (float x : q) std::printf("%.9g ", x);
        std::printf("\n");
    } else if (mode == "mbm" || mode == "scene") {
        auto envs = mode == "mbm" ? bcc_loaders::load_mbm(argv[2], 1000) : bcc_loaders::load_scene(argv[2], std::stoi(argv[3]));
        for (auto& e : envs) std::printf("%u %u %u\n", e.num_spheres, e.num_capsules, e.num_cuboids);
        // moved-from environments give up ownership
        ppln::collision::Environment<float> moved(std::move(envs[0]));
        std::printf("moved %d %d\n", (int)(envs[0].spheres == nullptr && envs[0].cuboids == nullptr), (int)moved.owns_memory);
    }
    return 0;
}
