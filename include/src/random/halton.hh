// Halton low-discrepancy sampler (drop-in for the reference header
// src/random/halton.hh: rng::Halton<dim>, next(), reset(), bases 3, 5, 7, ...).
//
// Each coordinate runs the incremental Halton recurrence on a fraction n / d
// (the algorithm given, e.g., in the Wikipedia article "Halton sequence"):
//   x = d - n;  if x == 1: n = 1, d = d * b   else: y = d / b (floor), while
//   x <= y: y = y / b (floor); n = (b + 1) y - x;   sample = n / d
// in single precision with floor after every division, as the reference does
// (its edge sets are reproduced bit for bit).  After max_iterations samples the
// state restarts with the bases rotated by one.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>

namespace rng {

template <std::size_t dim>
struct Halton {
    static constexpr std::size_t max_iterations = 1000000U;
    static constexpr std::array<float, 16> primes{3.F,  5.F,  7.F,  11.F, 13.F, 17.F, 19.F, 23.F,
                                                  29.F, 31.F, 37.F, 41.F, 43.F, 47.F, 53.F, 59.F};

    Halton() : Halton(bases()) {}
    explicit Halton(std::array<float, dim> b_in) : b_init(b_in), b(b_in) {
        n.fill(0.0f);
        d.fill(1.0f);
    }

    static std::array<float, dim> bases() {
        std::array<float, dim> a{};
        std::copy_n(primes.cbegin(), dim, a.begin());
        return a;
    }

    void rotate_bases() { std::rotate(b.begin(), b.begin() + 1, b.end()); }

    void reset() {
        iterations = 0;
        b = b_init;
        n.fill(0.0f);
        d.fill(1.0f);
    }

    std::array<float, dim> next() {
        if (++iterations > max_iterations) {
            n.fill(0.0f);
            d.fill(1.0f);
            iterations = 0;
            rotate_bases();
        }
        std::array<float, dim> out{};
        for (std::size_t i = 0; i < dim; ++i) {
            const float x = d[i] - n[i];
            if (x == 1.0f) {
                d[i] = std::floor(d[i] * b[i]);
                n[i] = 1.0f;
            } else {
                float y = std::floor(d[i] / b[i]);
                while (x <= y) y = std::floor(y / b[i]);
                n[i] = std::floor((b[i] + 1.0f) * y) - x;
            }
            out[i] = n[i] / d[i];
        }
        return out;
    }

    const std::array<float, dim> b_init;
    std::array<float, dim> b;
    std::array<float, dim> n;
    std::array<float, dim> d;
    std::size_t iterations = 0;
};

}  // namespace rng
