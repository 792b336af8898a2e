// bcc_device.cuh -- device-side building blocks of the B200 batch edge checker.
//
// Everything here is sm_100a CUDA written for this project.  The functions
// restate the reference's semantics (cited per function) in the data layout of
// this implementation:
//   * edges are discretised exactly as src/batch_cc.cu:96-129 does it;
//   * robot spheres come from a table-driven FK (robot_*.h) instead of the
//     reference's generated straight-line code;
//   * every environment primitive is one "rounded box" record, so one
//     branch-free predicate serves spheres, capsules and cuboids.
#pragma once

#include <cstdint>
#include <type_traits>
#include <utility>

#include <cuda_runtime.h>

namespace bcc {

constexpr int kLanes = 32;          // samples per reference round (src/batch_cc.cu:262)
constexpr int kBdim = kLanes - 1;   // bdim = blockDim.x - 1 (src/batch_cc.cu:82)
constexpr float kEnvInflate = 0.005f;  // robot radius inflation (src/utils.cuh:215)
constexpr float kCullMargin = 1e-4f;   // conservative slack of the AABB cull (m)
constexpr int kPrimF4 = 5;          // float4 words per primitive record

// ---------------------------------------------------------------------------
// Primitive record (5 x float4 = 80 bytes, 16-byte aligned for bulk copies):
//   w0 = centre.xyz, rho          (rounding radius)
//   w1 = axis1.xyz,  h1           (half-extent along axis1)
//   w2 = axis2.xyz,  h2
//   w3 = axis3.xyz,  h3
//   w4 = aabb half-size.xyz (incl. rho and cull margin), 0
// Squared distance from a point to the rounded box core is
//   sum_i max(|axis_i . d| - h_i, 0)^2,  d = point - centre,
// and the robot sphere (radius r, already inflated) collides when that sum is
// < (r + rho)^2.  This is the reference cuboid test (src/utils.cuh:159-178) for
// cuboids (rho = 0), the sphere test (:59-74) for spheres (h = 0), and the
// capsule test (:114-127) for capsules (h = (0, 0, len/2) along the capsule
// axis); all compare squared quantities with a strict < 0 like the reference.
// ---------------------------------------------------------------------------
// Squared distance from the sphere centre to the record's box core, and the
// record's rounding radius.
__device__ __forceinline__ float prim_core_d2(float4 s, const float4* __restrict__ rec, float* rho) {
    const float4 w0 = rec[0], w1 = rec[1], w2 = rec[2], w3 = rec[3];
    const float dx = s.x - w0.x, dy = s.y - w0.y, dz = s.z - w0.z;
    const float p1 = fmaf(w1.x, dx, fmaf(w1.y, dy, w1.z * dz));
    const float p2 = fmaf(w2.x, dx, fmaf(w2.y, dy, w2.z * dz));
    const float p3 = fmaf(w3.x, dx, fmaf(w3.y, dy, w3.z * dz));
    const float e1 = fmaxf(fabsf(p1) - w1.w, 0.0f);
    const float e2 = fmaxf(fabsf(p2) - w2.w, 0.0f);
    const float e3 = fmaxf(fabsf(p3) - w3.w, 0.0f);
    *rho = w0.w;
    return fmaf(e1, e1, fmaf(e2, e2, e3 * e3));
}

__device__ __forceinline__ bool sphere_hits_prim(float4 s, const float4* __restrict__ rec) {
    float rho;
    const float sum = prim_core_d2(s, rec, &rho);
    const float rr = s.w + rho;
    return sum - rr * rr < 0.0f;
}

// ---------------------------------------------------------------------------
// Reference discretisation, bit-exact (src/batch_cc.cu:96-129).  Explicit
// intrinsics pin the rounding of every step: the squared length accumulates
// with fused multiply-adds, sqrt and divides are IEEE, lane t's first sample is
// fma(delta, t*n, start) and each further round adds delta once.
// ---------------------------------------------------------------------------
template <int DOF>
__device__ __forceinline__ int edge_steps(const float* s, const float* e, int resolution) {
    float ans = 0.0f;
#pragma unroll
    for (int j = 0; j < DOF; ++j) {
        const float d = __fsub_rn(s[j], e[j]);
        ans = __fmaf_rn(d, d, ans);
    }
    const float dist = __fsqrt_rn(ans);
    const float nf = fmaxf(ceilf(__fmul_rn(__fdiv_rn(dist, (float)kBdim), (float)resolution)), 1.0f);
    return (int)nf;
}

template <int DOF>
__device__ __forceinline__ void edge_sample(const float* s, const float* e, int n, int k, float* q) {
    const int lane = k / n;
    const int round = k - lane * n;
    const float denom = (float)(kBdim * n);
    const float tn = (float)(lane * n);
#pragma unroll
    for (int j = 0; j < DOF; ++j) {
        const float delta = __fdiv_rn(__fsub_rn(e[j], s[j]), denom);
        float c = __fmaf_rn(delta, tn, s[j]);
        for (int i = 0; i < round; ++i) c = __fadd_rn(c, delta);
        q[j] = c;
    }
}

// Rank r of the reference's check order -> sample index k: round r / 32,
// lane r % 32 checks sample k = lane * n + round (src/batch_cc.cu:113-129).
__device__ __forceinline__ int reference_rank_to_sample(int r, int n) {
    return (r & (kLanes - 1)) * n + (r >> 5);
}

// ---------------------------------------------------------------------------
// Table-driven forward kinematics over a kinematic tree:
//   frame k+1 = frame joint_parent[k] * F_k * J_k(q_k),
// J = Rz(q) (revolute, type 0) or Tz(q) (prismatic, type 1), F_k from
// M::joint_tf; sphere centre = R_f * local + p_f.  Scalar type T is float for
// robots whose reference FK is float code (Panda) and double where the
// reference evaluates its FK in double (Fetch, Baxter); centres are rounded to
// float either way, as the reference does when it passes them to the tests.
// Each sphere is emitted right after its frame is known, so a frame stays
// live only while later joints or spheres still need it.
// ---------------------------------------------------------------------------
template <class M, class T>
struct Frames {
    T R[M::dof + 1][9];
    T p[M::dof + 1][3];
};

template <class M, int S, class T>
__device__ __forceinline__ float4 fk_sphere(const Frames<M, T>& F) {
    constexpr int f = M::sphere_frame[S];
    constexpr T lx = (T)M::sphere_local[S][0];
    constexpr T ly = (T)M::sphere_local[S][1];
    constexpr T lz = (T)M::sphere_local[S][2];
    float4 c;
    c.x = (float)(F.R[f][0] * lx + F.R[f][1] * ly + F.R[f][2] * lz + F.p[f][0]);
    c.y = (float)(F.R[f][3] * lx + F.R[f][4] * ly + F.R[f][5] * lz + F.p[f][1]);
    c.z = (float)(F.R[f][6] * lx + F.R[f][7] * ly + F.R[f][8] * lz + F.p[f][2]);
    c.w = M::sphere_radius[S];
    return c;
}

// Sample table layout: rows in tiles of M::table_tile rows, sphere-major inside
// a tile (a tile of 1 is plain row-major).  With tiles of 32, 32 consecutive
// rows of one sphere are 512 contiguous bytes and the FK kernel's warp (32
// consecutive rows) writes each sphere with one coalesced store; row-major keeps
// a row's bounds and leaves together for the check kernel's reads.
constexpr int kMaxTableTile = 32;  // hosts round row counts up to this

template <class M>
__host__ __device__ __forceinline__ size_t table_index(size_t row, int s) {
    constexpr int TT = M::table_tile;
    return ((row / TT) * M::num_spheres + s) * TT + (row % TT);
}

// Write every sphere attached to frame FR into its sample-table position; `out`
// points at the row's first sphere, spheres M::table_tile float4 apart.
template <class M, int FR, int S, class T>
__device__ __forceinline__ void emit_one(const Frames<M, T>& F, float4* __restrict__ out) {
    if constexpr (M::sphere_frame[S] == FR) {
        constexpr int pos = M::table_pos[S];
        out[pos * M::table_tile] = fk_sphere<M, S, T>(F);
    }
}
template <class M, int FR, class T, int... S>
__device__ __forceinline__ void emit_frame(const Frames<M, T>& F, float4* __restrict__ out,
                                           std::integer_sequence<int, S...>) {
    (emit_one<M, FR, S, T>(F, out), ...);
}

__device__ __forceinline__ void sin_cos(float q, float* s, float* c) { sincosf(q, s, c); }
__device__ __forceinline__ void sin_cos(double q, double* s, double* c) { sincos(q, s, c); }

// One joint: compile-time constants of F_K are folded into the multiply-adds.
template <class M, int K, class T>
struct FkJoint {
    __device__ __forceinline__ static void run(const float* q, Frames<M, T>& F, float4* __restrict__ out) {
        constexpr int P = M::joint_parent[K];
        static_assert(P <= K, "joints must follow their parents");
        constexpr T f[12] = {
            (T)M::joint_tf[K][0], (T)M::joint_tf[K][1], (T)M::joint_tf[K][2],
            (T)M::joint_tf[K][3], (T)M::joint_tf[K][4], (T)M::joint_tf[K][5],
            (T)M::joint_tf[K][6], (T)M::joint_tf[K][7], (T)M::joint_tf[K][8],
            (T)M::joint_tf[K][9], (T)M::joint_tf[K][10], (T)M::joint_tf[K][11]};
        T A[9];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int b = 0; b < 3; ++b)
                A[a * 3 + b] = F.R[P][a * 3 + 0] * f[0 * 4 + b] + F.R[P][a * 3 + 1] * f[1 * 4 + b] +
                               F.R[P][a * 3 + 2] * f[2 * 4 + b];
            F.p[K + 1][a] = F.R[P][a * 3 + 0] * f[3] + F.R[P][a * 3 + 1] * f[7] +
                            F.R[P][a * 3 + 2] * f[11] + F.p[P][a];
        }
        const T qk = (T)q[K];
        if constexpr (M::joint_type[K] == 0) {
            T sq, cq;
            sin_cos(qk, &sq, &cq);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                F.R[K + 1][a * 3 + 0] = A[a * 3 + 0] * cq + A[a * 3 + 1] * sq;
                F.R[K + 1][a * 3 + 1] = A[a * 3 + 1] * cq - A[a * 3 + 0] * sq;
                F.R[K + 1][a * 3 + 2] = A[a * 3 + 2];
            }
        } else {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
#pragma unroll
                for (int b = 0; b < 3; ++b) F.R[K + 1][a * 3 + b] = A[a * 3 + b];
                F.p[K + 1][a] += A[a * 3 + 2] * qk;
            }
        }
        emit_frame<M, K + 1, T>(F, out, std::make_integer_sequence<int, M::num_spheres>{});
        FkJoint<M, K + 1, T>::run(q, F, out);
    }
};

template <class M, class T>
struct FkJoint<M, M::dof, T> {
    __device__ __forceinline__ static void run(const float*, Frames<M, T>&, float4* __restrict__) {}
};

// All sphere centres of configuration q into out[table_pos[s] * table_tile].
template <class M>
__device__ __forceinline__ void fk_spheres(const float* q, float4* __restrict__ out) {
    using T = typename std::conditional<M::fk_precision == 64, double, float>::type;
    Frames<M, T> F;
#pragma unroll
    for (int i = 0; i < 9; ++i) F.R[0][i] = (i % 4 == 0) ? T(1) : T(0);
    F.p[0][0] = F.p[0][1] = F.p[0][2] = T(0);
    emit_frame<M, 0, T>(F, out, std::make_integer_sequence<int, M::num_spheres>{});
    FkJoint<M, 0, T>::run(q, F, out);
}

// Bounded mbarrier wait: gives up after `limit` polls and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    const uint32_t addr = (uint32_t)__cvta_generic_to_shared(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    const uint32_t addr = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

// One thread: expect `bytes` on the barrier and start a 1-D bulk copy
// global -> shared (no multicast).  src/dst 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
        "l"(src), "r"(bytes), "r"(b)
        : "memory");
}

}  // namespace bcc
