/*
 * oracle.cpp -- CPU restatement of the reference batch edge collision check.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path links, loads or calls
 * this file; tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py use it as the checker and as the timed CPU baseline.
 *
 * What it restates (reference paths relative to the reference project root):
 *  - edge discretisation, FP32 and bit-exact: src/batch_cc.cu:96-129
 *      n     = max(ceil(sqrt(sum (s-e)^2) / 31 * resolution), 1)
 *      delta = (e - s) / (31 * n)
 *      lane t (0..31), round i (0..n-1): q = fma(delta, t*n, s) + i * delta,
 *      the i additions done one at a time in FP32 (src/batch_cc.cu:126-128);
 *  - per-configuration check fkcc<Robot> (src/utils.cuh:342-5443 for Panda):
 *      the reference's environment groups (the ref_env_* tables) in order,
 *      bounding sphere gate then leaf spheres
 *      (:806-1190, link0 never env-checked), then self groups, bound pair gate
 *      then leaf pairs (:1192-5440); any hit = collision;
 *  - environment scan sphere_environment_in_collision (src/utils.cuh:213-245):
 *      robot radius + 0.005 m; spheres, capsules, z-capsules, cuboids,
 *      z-cuboids in that order; cylinders never read; strict < 0 tests
 *      (predicates at src/utils.cuh:59-88, :114-210);
 *  - edge verdict = any colliding sample among the 32 n samples, rounds of 32
 *      with early exit (src/batch_cc.cu:118-129); results [edge][env].
 * Forward kinematics is evaluated from the robot's chain tables (robot_*.h),
 * which reproduce the reference's generated FK to FP64 rounding.
 *
 * Two arithmetic modes of the check: FP64 (the adjudication oracle) and FP32
 * (the timed CPU baseline, the reference's arithmetic width).  A third entry
 * computes the FP64 signed penetration of a pair, the quantity mismatches are
 * adjudicated on: for one sample
 *   env_pen  = max_g min(pen(bound_g), max_leaf pen(leaf))
 *   self_pen = max_g min(pen(bound pair_g), max_pair pen(leaf pair))
 * with pen > 0 meaning penetration in metres; the pair's value is the maximum
 * over its samples.  A verdict disagreement is tolerated only when
 * |pen| <= 1e-5 m.
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "../include/bcc.h"
#include "../batch-cc_b200/csrc/robot_baxter.h"
#include "../batch-cc_b200/csrc/robot_fetch.h"
#include "../batch-cc_b200/csrc/robot_panda.h"

namespace {

constexpr int kLanes = 32;      // reference block size (src/batch_cc.cu:262)
constexpr int kBdim = kLanes - 1;  // bdim = blockDim.x - 1 (src/batch_cc.cu:82)

struct EnvView {
    uint32_t n[5];  // spheres, capsules, z-capsules, cuboids, z-cuboids
    const float* rec[5];
};

std::vector<EnvView> make_views(const bcc_env_soa* e) {
    std::vector<EnvView> v(e->num_envs);
    const uint32_t* cnt[5] = {e->num_spheres, e->num_capsules, e->num_z_capsules,
                              e->num_cuboids, e->num_z_cuboids};
    const float* base[5] = {e->spheres, e->capsules, e->z_capsules, e->cuboids, e->z_cuboids};
    const int width[5] = {4, 8, 8, 15, 15};
    size_t off[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < e->num_envs; ++i) {
        for (int k = 0; k < 5; ++k) {
            uint32_t c = cnt[k] ? cnt[k][i] : 0;
            v[i].n[k] = c;
            v[i].rec[k] = c ? base[k] + off[k] * width[k] : nullptr;
            off[k] += c;
        }
    }
    return v;
}

// ---------------------------------------------------------------- discretisation
struct Disc {
    int n;
    float start[16];
    float delta[16];
};

Disc discretise(const float* s, const float* e, int dof, int resolution) {
    Disc d;
    float ans = 0.0f;
    for (int j = 0; j < dof; ++j) {
        float diff = s[j] - e[j];
        ans = std::fmaf(diff, diff, ans);
    }
    float dist = std::sqrt(ans);
    float nf = std::fmax(std::ceil((dist / (float)kBdim) * (float)resolution), 1.0f);
    d.n = (int)nf;
    for (int j = 0; j < dof; ++j) {
        d.start[j] = s[j];
        d.delta[j] = (e[j] - s[j]) / (float)(kBdim * d.n);
    }
    return d;
}

inline void sample_q(const Disc& d, int dof, int lane, int round, float* q) {
    for (int j = 0; j < dof; ++j) {
        float c = std::fmaf(d.delta[j], (float)(lane * d.n), d.start[j]);
        for (int i = 0; i < round; ++i) c = c + d.delta[j];
        q[j] = c;
    }
}

// ---------------------------------------------------------------- kinematics
// Tree FK from the robot tables: frame k+1 = frame parent(k) * F_k * J_k(q_k),
// J = Rz (revolute) or Tz (prismatic); evaluated in T.
template <class M, class T>
void tree_fk(const float* qf, T (*c)[3]) {
    T R[M::dof + 1][3][3];
    T p[M::dof + 1][3];
    for (int a = 0; a < 3; ++a) {
        for (int b = 0; b < 3; ++b) R[0][a][b] = (a == b) ? T(1) : T(0);
        p[0][a] = T(0);
    }
    for (int k = 0; k < M::dof; ++k) {
        const double* F = M::joint_tf[k];
        const int P = M::joint_parent[k];
        T A[3][3];
        for (int a = 0; a < 3; ++a) {
            for (int b = 0; b < 3; ++b)
                A[a][b] = R[P][a][0] * T(F[0 * 4 + b]) + R[P][a][1] * T(F[1 * 4 + b]) +
                          R[P][a][2] * T(F[2 * 4 + b]);
            p[k + 1][a] = R[P][a][0] * T(F[3]) + R[P][a][1] * T(F[7]) + R[P][a][2] * T(F[11]) +
                          p[P][a];
        }
        T q = T(qf[k]);
        if (M::joint_type[k] == 0) {
            T cq = std::cos(q), sq = std::sin(q);
            for (int a = 0; a < 3; ++a) {
                R[k + 1][a][0] = A[a][0] * cq + A[a][1] * sq;
                R[k + 1][a][1] = A[a][1] * cq - A[a][0] * sq;
                R[k + 1][a][2] = A[a][2];
            }
        } else {
            for (int a = 0; a < 3; ++a) {
                for (int b = 0; b < 3; ++b) R[k + 1][a][b] = A[a][b];
                p[k + 1][a] += A[a][2] * q;
            }
        }
    }
    for (int s = 0; s < M::num_spheres; ++s) {
        int f = M::sphere_frame[s];
        const double* l = M::sphere_local[s];
        for (int a = 0; a < 3; ++a)
            c[s][a] = R[f][a][0] * T(l[0]) + R[f][a][1] * T(l[1]) + R[f][a][2] * T(l[2]) + p[f][a];
    }
}

// Sphere centres in T.  Where the reference evaluates the robot's FK in double
// (Fetch, Baxter: `auto X = q * 0.5; sin(X)` promotes) and passes the centres
// to the float tests, the FP32 mode does the same: double FK, rounded to float.
template <class M, class T>
void forward_kinematics(const float* qf, T (*c)[3]) {
    if (M::fk_precision == 64 && sizeof(T) < sizeof(double)) {
        double cd[M::num_spheres][3];
        tree_fk<M, double>(qf, cd);
        for (int s = 0; s < M::num_spheres; ++s)
            for (int a = 0; a < 3; ++a) c[s][a] = T(cd[s][a]);
    } else {
        tree_fk<M, T>(qf, c);
    }
}

// ---------------------------------------------------------------- predicates
// Each returns the reference's "squared" test value; < 0 means collision.
template <class T>
inline T clamp01(T v) {  // fmaxf(fminf(v, 1), 0): a NaN input yields 1 (src/utils.cuh:52-55)
    return std::fmax(std::fmin(v, T(1)), T(0));
}

template <class T>
inline T t_sphere(const float* s, T x, T y, T z, T r) {
    T dx = x - T(s[0]), dy = y - T(s[1]), dz = z - T(s[2]);
    T rs = r + T(s[3]);
    return dx * dx + dy * dy + dz * dz - rs * rs;
}
template <class T>
inline T t_capsule(const float* c, T x, T y, T z, T r) {
    T dot = (x - T(c[0])) * T(c[3]) + (y - T(c[1])) * T(c[4]) + (z - T(c[2])) * T(c[5]);
    T cdf = clamp01(dot * T(c[7]));
    T px = T(c[0]) + T(c[3]) * cdf, py = T(c[1]) + T(c[4]) * cdf, pz = T(c[2]) + T(c[5]) * cdf;
    T dx = x - px, dy = y - py, dz = z - pz;
    T rs = r + T(c[6]);
    return dx * dx + dy * dy + dz * dz - rs * rs;
}
template <class T>
inline T t_zcapsule(const float* c, T x, T y, T z, T r) {
    T dot = (z - T(c[2])) * T(c[5]);
    T cdf = clamp01(dot * T(c[7]));
    T dx = x - T(c[0]), dy = y - T(c[1]), dz = z - (T(c[2]) + T(c[5]) * cdf);
    T rs = r + T(c[6]);
    return dx * dx + dy * dy + dz * dz - rs * rs;
}
template <class T>
inline T t_cuboid(const float* b, T x, T y, T z, T rsq) {
    T xs = x - T(b[0]), ys = y - T(b[1]), zs = z - T(b[2]);
    T a1 = std::fmax(T(0), std::fabs(T(b[3]) * xs + T(b[4]) * ys + T(b[5]) * zs) - T(b[12]));
    T a2 = std::fmax(T(0), std::fabs(T(b[6]) * xs + T(b[7]) * ys + T(b[8]) * zs) - T(b[13]));
    T a3 = std::fmax(T(0), std::fabs(T(b[9]) * xs + T(b[10]) * ys + T(b[11]) * zs) - T(b[14]));
    return a1 * a1 + a2 * a2 + a3 * a3 - rsq;
}
template <class T>
inline T t_zcuboid(const float* b, T x, T y, T z, T rsq) {
    T xs = x - T(b[0]), ys = y - T(b[1]), zs = z - T(b[2]);
    T a1 = std::fmax(T(0), std::fabs(T(b[3]) * xs + T(b[4]) * ys) - T(b[12]));
    T a2 = std::fmax(T(0), std::fabs(T(b[6]) * xs + T(b[7]) * ys) - T(b[13]));
    T a3 = std::fmax(T(0), std::fabs(zs) - T(b[14]));
    return a1 * a1 + a2 * a2 + a3 * a3 - rsq;
}

// sphere_environment_in_collision (src/utils.cuh:213-245)
template <class T>
bool env_hit(const EnvView& e, T x, T y, T z, T r) {
    r = r + T(0.005);
    const T rsq = r * r;
    for (uint32_t i = 0; i < e.n[0]; ++i)
        if (t_sphere<T>(e.rec[0] + 4 * i, x, y, z, r) < 0) return true;
    for (uint32_t i = 0; i < e.n[1]; ++i)
        if (t_capsule<T>(e.rec[1] + 8 * i, x, y, z, r) < 0) return true;
    for (uint32_t i = 0; i < e.n[2]; ++i)
        if (t_zcapsule<T>(e.rec[2] + 8 * i, x, y, z, r) < 0) return true;
    for (uint32_t i = 0; i < e.n[3]; ++i)
        if (t_cuboid<T>(e.rec[3] + 15 * i, x, y, z, rsq) < 0) return true;
    for (uint32_t i = 0; i < e.n[4]; ++i)
        if (t_zcuboid<T>(e.rec[4] + 15 * i, x, y, z, rsq) < 0) return true;
    return false;
}

// Signed penetration (m) of an inflated robot sphere into the environment (max over
// primitives); the FP64 counterpart of the squared tests above.
double env_pen(const EnvView& e, double x, double y, double z, double r) {
    r = r + 0.005;
    double best = -std::numeric_limits<double>::infinity();
    auto upd = [&](double dist) { best = std::max(best, -dist); };
    for (uint32_t i = 0; i < e.n[0]; ++i) {
        const float* s = e.rec[0] + 4 * i;
        double dx = x - s[0], dy = y - s[1], dz = z - s[2];
        upd(std::sqrt(dx * dx + dy * dy + dz * dz) - (r + s[3]));
    }
    for (int k = 1; k <= 2; ++k)
        for (uint32_t i = 0; i < e.n[k]; ++i) {
            const float* c = e.rec[k] + 8 * i;
            double t = k == 1 ? t_capsule<double>(c, x, y, z, 0.0) : t_zcapsule<double>(c, x, y, z, 0.0);
            // t = d^2 - c.r^2 with r = 0 passed in; recover d.
            double d = std::sqrt(std::max(0.0, t + double(c[6]) * double(c[6])));
            upd(d - (r + c[6]));
        }
    for (int k = 3; k <= 4; ++k)
        for (uint32_t i = 0; i < e.n[k]; ++i) {
            const float* b = e.rec[k] + 15 * i;
            double t = k == 3 ? t_cuboid<double>(b, x, y, z, 0.0) : t_zcuboid<double>(b, x, y, z, 0.0);
            upd(std::sqrt(std::max(0.0, t)) - r);
        }
    return best;
}

template <class M, class T>
bool config_collides(const EnvView& e, const float* q) {
    T c[M::num_spheres][3];
    forward_kinematics<M, T>(q, c);
    for (int g = 0; g < M::num_ref_env_groups; ++g) {
        int b = M::ref_env_bound[g];
        if (!env_hit<T>(e, c[b][0], c[b][1], c[b][2], T(M::sphere_radius[b]))) continue;
        for (int k = M::ref_env_leaf_begin[g]; k < M::ref_env_leaf_begin[g + 1]; ++k) {
            int s = M::ref_env_leaves[k];
            if (env_hit<T>(e, c[s][0], c[s][1], c[s][2], T(M::sphere_radius[s]))) return true;
        }
    }
    auto self = [&](int a, int b) {
        T dx = c[a][0] - c[b][0], dy = c[a][1] - c[b][1], dz = c[a][2] - c[b][2];
        T rs = T(M::sphere_radius[a]) + T(M::sphere_radius[b]);
        return dx * dx + dy * dy + dz * dz - rs * rs < 0;
    };
    for (int g = 0; g < M::num_self_groups; ++g) {
        if (!self(M::self_bound[g][0], M::self_bound[g][1])) continue;
        for (int k = M::self_pair_begin[g]; k < M::self_pair_begin[g + 1]; ++k)
            if (self(M::self_pairs[k][0], M::self_pairs[k][1])) return true;
    }
    return false;
}

template <class M>
double config_pen(const EnvView& e, const float* q) {
    double c[M::num_spheres][3];
    forward_kinematics<M, double>(q, c);
    const double ninf = -std::numeric_limits<double>::infinity();
    double best = ninf;
    for (int g = 0; g < M::num_ref_env_groups; ++g) {
        int b = M::ref_env_bound[g];
        double gp = env_pen(e, c[b][0], c[b][1], c[b][2], M::sphere_radius[b]);
        double lp = ninf;
        for (int k = M::ref_env_leaf_begin[g]; k < M::ref_env_leaf_begin[g + 1]; ++k) {
            int s = M::ref_env_leaves[k];
            lp = std::max(lp, env_pen(e, c[s][0], c[s][1], c[s][2], M::sphere_radius[s]));
        }
        best = std::max(best, std::min(gp, lp));
    }
    auto self = [&](int a, int b) {
        double dx = c[a][0] - c[b][0], dy = c[a][1] - c[b][1], dz = c[a][2] - c[b][2];
        return double(M::sphere_radius[a]) + double(M::sphere_radius[b]) -
               std::sqrt(dx * dx + dy * dy + dz * dz);
    };
    for (int g = 0; g < M::num_self_groups; ++g) {
        double gp = self(M::self_bound[g][0], M::self_bound[g][1]);
        double lp = ninf;
        for (int k = M::self_pair_begin[g]; k < M::self_pair_begin[g + 1]; ++k)
            lp = std::max(lp, self(M::self_pairs[k][0], M::self_pairs[k][1]));
        best = std::max(best, std::min(gp, lp));
    }
    return best;
}

// Algorithmic FLOPs of one fkcc call in the reference's literal order: FK, then
// each sphere_environment_in_collision call (2 for the inflation + per tested
// primitive 11 sphere / 28 capsule / 18 z-capsule / 33 cuboid / 24 z-cuboid,
// stopping at the first hit), then 11 per self test; returns the verdict.
constexpr double kFlopPrim[5] = {11.0, 28.0, 18.0, 33.0, 24.0};

template <class M>
bool config_flops(const EnvView& e, const float* q, double& flops) {
    float c[M::num_spheres][3];
    forward_kinematics<M, float>(q, c);
    flops += double(M::fk_flops);
    auto scan = [&](int s) {
        float x = c[s][0], y = c[s][1], z = c[s][2];
        float r = M::sphere_radius[s] + 0.005f;
        const float rsq = r * r;
        flops += 2.0;
        for (int k = 0; k < 5; ++k)
            for (uint32_t i = 0; i < e.n[k]; ++i) {
                flops += kFlopPrim[k];
                float t;
                switch (k) {
                    case 0: t = t_sphere<float>(e.rec[0] + 4 * i, x, y, z, r); break;
                    case 1: t = t_capsule<float>(e.rec[1] + 8 * i, x, y, z, r); break;
                    case 2: t = t_zcapsule<float>(e.rec[2] + 8 * i, x, y, z, r); break;
                    case 3: t = t_cuboid<float>(e.rec[3] + 15 * i, x, y, z, rsq); break;
                    default: t = t_zcuboid<float>(e.rec[4] + 15 * i, x, y, z, rsq); break;
                }
                if (t < 0) return true;
            }
        return false;
    };
    for (int g = 0; g < M::num_ref_env_groups; ++g) {
        if (!scan(M::ref_env_bound[g])) continue;
        for (int k = M::ref_env_leaf_begin[g]; k < M::ref_env_leaf_begin[g + 1]; ++k)
            if (scan(M::ref_env_leaves[k])) return true;
    }
    auto self = [&](int a, int b) {
        flops += 11.0;
        float dx = c[a][0] - c[b][0], dy = c[a][1] - c[b][1], dz = c[a][2] - c[b][2];
        float rs = M::sphere_radius[a] + M::sphere_radius[b];
        return dx * dx + dy * dy + dz * dz - rs * rs < 0;
    };
    for (int g = 0; g < M::num_self_groups; ++g) {
        if (!self(M::self_bound[g][0], M::self_bound[g][1])) continue;
        for (int k = M::self_pair_begin[g]; k < M::self_pair_begin[g + 1]; ++k)
            if (self(M::self_pairs[k][0], M::self_pairs[k][1])) return true;
    }
    return false;
}

// Reference plain order: all 32 lanes of a round are evaluated, the pair stops
// after the first round with a hit.
template <class M>
double pair_flops(const EnvView& e, const float* edge, int resolution, uint8_t* verdict) {
    Disc d = discretise(edge, edge + M::dof, M::dof, resolution);
    float q[16];
    double flops = 0.0;
    for (int i = 0; i < d.n; ++i) {
        bool any = false;
        for (int t = 0; t < kLanes; ++t) {
            sample_q(d, M::dof, t, i, q);
            any |= config_flops<M>(e, q, flops);
        }
        if (any) {
            *verdict = 1;
            return flops;
        }
    }
    *verdict = 0;
    return flops;
}

// Reference pair verdict: rounds of 32 lanes, early exit after a colliding round.
template <class M, class T>
uint8_t pair_verdict(const EnvView& e, const float* edge, int resolution) {
    Disc d = discretise(edge, edge + M::dof, M::dof, resolution);
    float q[16];
    for (int i = 0; i < d.n; ++i)
        for (int t = 0; t < kLanes; ++t) {
            sample_q(d, M::dof, t, i, q);
            if (config_collides<M, T>(e, q)) return 1;
        }
    return 0;
}

template <class F>
void parallel_for(int64_t n, int nthreads, F f) {
    if (nthreads <= 1 || n < 2) {
        for (int64_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int64_t> next(0);
    std::vector<std::thread> th;
    for (int w = 0; w < nthreads; ++w)
        th.emplace_back([&] {
            for (;;) {
                int64_t i0 = next.fetch_add(64);
                if (i0 >= n) break;
                int64_t i1 = std::min(n, i0 + 64);
                for (int64_t i = i0; i < i1; ++i) f(i);
            }
        });
    for (auto& t : th) t.join();
}

template <class M>
int check_impl(const bcc_env_soa* envs, const float* edges, int E, int res, int precision,
               int nthreads, uint8_t* out) {
    auto views = make_views(envs);
    const int64_t N = envs->num_envs;
    parallel_for(N * (int64_t)E, nthreads, [&](int64_t idx) {
        int64_t e = idx / N, v = idx % N;
        const float* edge = edges + e * 2 * M::dof;
        out[idx] = precision == 32 ? pair_verdict<M, float>(views[v], edge, res)
                                   : pair_verdict<M, double>(views[v], edge, res);
    });
    return 0;
}

template <class M>
int pen_impl(const bcc_env_soa* envs, const float* edges, int res, const int64_t* pairs, int K,
             int nthreads, double* pen, int32_t* arg) {
    auto views = make_views(envs);
    parallel_for(K, nthreads, [&](int64_t k) {
        int64_t e = pairs[2 * k], v = pairs[2 * k + 1];
        const float* edge = edges + e * 2 * M::dof;
        Disc d = discretise(edge, edge + M::dof, M::dof, res);
        float q[16];
        double best = -std::numeric_limits<double>::infinity();
        int32_t bi = -1;
        for (int t = 0; t < kLanes; ++t)
            for (int i = 0; i < d.n; ++i) {
                sample_q(d, M::dof, t, i, q);
                double p = config_pen<M>(views[v], q);
                if (p > best || bi < 0) {
                    best = p;
                    bi = t * d.n + i;
                }
            }
        pen[k] = best;
        if (arg) arg[k] = bi;
    });
    return 0;
}

}  // namespace

// Runs f(Model{}) for the robot's model; `fallback` for an unknown robot.
template <class R, class F>
R with_robot(int robot, R fallback, F&& f) {
    switch (robot) {
        case BCC_ROBOT_PANDA: return f(bcc::PandaModel{});
        case BCC_ROBOT_FETCH: return f(bcc::FetchModel{});
        case BCC_ROBOT_BAXTER: return f(bcc::BaxterModel{});
        default: return fallback;
    }
}

extern "C" {

int orc_robot_dof(int robot) {
    return with_robot(robot, -1, [](auto m) { return decltype(m)::dof; });
}

int orc_robot_num_spheres(int robot) {
    return with_robot(robot, -1, [](auto m) { return decltype(m)::num_spheres; });
}

int orc_edge_n(const float* start, const float* end, int dof, int resolution) {
    return discretise(start, end, dof, resolution).n;
}

// Samples in index order k = lane * n + round (t_k = k / (31 n)); out holds 32 n rows.
int orc_edge_samples(const float* start, const float* end, int dof, int resolution, float* out) {
    Disc d = discretise(start, end, dof, resolution);
    for (int t = 0; t < kLanes; ++t)
        for (int i = 0; i < d.n; ++i) sample_q(d, dof, t, i, out + (int64_t)(t * d.n + i) * dof);
    return d.n;
}

// Sphere centres [num_spheres][3] of a configuration, FP64 tree FK.
int orc_fk(int robot, const float* q, double* centres) {
    return with_robot(robot, -1, [&](auto m) {
        using M = decltype(m);
        forward_kinematics<M, double>(q, (double(*)[3])centres);
        return 0;
    });
}

// One configuration against one environment (literal fkcc semantics); 1 = collision.
int orc_config_collides(const bcc_env_soa* envs, int env, int robot, const float* q, int precision) {
    return with_robot(robot, -1, [&](auto m) {
        using M = decltype(m);
        auto views = make_views(envs);
        return (int)(precision == 32 ? config_collides<M, float>(views[env], q)
                                     : config_collides<M, double>(views[env], q));
    });
}

double orc_config_pen(const bcc_env_soa* envs, int env, int robot, const float* q) {
    return with_robot(robot, std::nan(""), [&](auto m) {
        using M = decltype(m);
        auto views = make_views(envs);
        return config_pen<M>(views[env], q);
    });
}

// Verdicts of every (env, edge) pair, results[edge][env]; precision 64 or 32.
int orc_check(const bcc_env_soa* envs, int robot, const float* edges, int num_edges, int resolution,
              int precision, int nthreads, uint8_t* out) {
    return with_robot(robot, -1, [&](auto m) {
        using M = decltype(m);
        return check_impl<M>(envs, edges, num_edges, resolution, precision, nthreads, out);
    });
}

// FP64 penetration of listed (edge, env) pairs; arg = sample index k of the maximum.
int orc_pair_pen(const bcc_env_soa* envs, int robot, const float* edges, int resolution,
                 const int64_t* pairs, int num_pairs, int nthreads, double* pen, int32_t* arg) {
    return with_robot(robot, -1, [&](auto m) {
        using M = decltype(m);
        return pen_impl<M>(envs, edges, resolution, pairs, num_pairs, nthreads, pen, arg);
    });
}

// Algorithmic FLOPs (reference plain order) of listed (edge, env) pairs.
int orc_pair_flops(const bcc_env_soa* envs, int robot, const float* edges, int resolution,
                   const int64_t* pairs, int num_pairs, int nthreads, double* flops, uint8_t* verdict) {
    return with_robot(robot, -1, [&](auto m) {
        using M = decltype(m);
        auto views = make_views(envs);
        parallel_for(num_pairs, nthreads, [&](int64_t k) {
            int64_t e = pairs[2 * k], v = pairs[2 * k + 1];
            flops[k] = pair_flops<M>(views[v], edges + e * 2 * M::dof, resolution, verdict + k);
        });
        return 0;
    });
}

// Per-sample verdicts of listed (edge, env) pairs: out[k * max_samples + j] = 1
// when sample j (index order j = lane * n + round) of pair k collides, 0 when
// it is free, 2 past the pair's 32 n samples (or when 32 n > max_samples).
int orc_pair_samples(const bcc_env_soa* envs, int robot, const float* edges, int resolution,
                     const int64_t* pairs, int num_pairs, int max_samples, int precision, int nthreads,
                     uint8_t* out) {
    return with_robot(robot, -1, [&](auto m) {
        using M = decltype(m);
        auto views = make_views(envs);
        parallel_for(num_pairs, nthreads, [&](int64_t k) {
            int64_t e = pairs[2 * k], v = pairs[2 * k + 1];
            const float* edge = edges + e * 2 * M::dof;
            Disc d = discretise(edge, edge + M::dof, M::dof, resolution);
            uint8_t* o = out + k * (int64_t)max_samples;
            std::fill(o, o + max_samples, (uint8_t)2);
            if ((int64_t)kLanes * d.n > max_samples) return;
            float q[16];
            for (int t = 0; t < kLanes; ++t)
                for (int i = 0; i < d.n; ++i) {
                    sample_q(d, M::dof, t, i, q);
                    o[t * d.n + i] = precision == 32 ? (uint8_t)config_collides<M, float>(views[v], q)
                                                     : (uint8_t)config_collides<M, double>(views[v], q);
                }
        });
        return 0;
    });
}

}  // extern "C"
