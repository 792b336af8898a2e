// Draws from rng::Halton<dim> for dim = 7, 8, 14 (Panda, Fetch, Baxter):
// 1,000,010 draws each -- past the sampler's restart after max_iterations --
// hashed bit for bit (FNV-1a over the float32 words), plus the rows around the
// start and the restart.  Compiled against either the reference's header or
// the drop-in (tests/golden/make_halton.py, tests/test_dropin.py): the include
// path decides which "src/random/halton.hh" is used.
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>

#include "src/random/halton.hh"

template <std::size_t dim>
void run() {
    rng::Halton<dim> h;
    uint64_t hash = 1469598103934665603ull;
    const long total = 1000010;
    std::printf("dim %zu\n", dim);
    for (long i = 0; i < total; ++i) {
        const std::array<float, dim> v = h.next();
        for (float x : v) {
            uint32_t u;
            std::memcpy(&u, &x, 4);
            for (int k = 0; k < 4; ++k) {
                hash ^= (u >> (8 * k)) & 0xffu;
                hash *= 1099511628211ull;
            }
        }
        if (i < 4 || (i >= 999998 && i < 1000004)) {
            std::printf("row %ld", i);
            for (float x : v) std::printf(" %a", x);
            std::printf("\n");
        }
    }
    std::printf("fnv1a64 %016llx\n", (unsigned long long)hash);
}

int main() {
    run<7>();
    run<8>();
    run<14>();
    return 0;
}
