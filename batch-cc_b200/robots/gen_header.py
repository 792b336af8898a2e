"""Write the C++/CUDA robot-model header from an extracted robot JSON.

The header holds plain constexpr tables (joint fixed transforms, parents and
types, sphere
frames/offsets/radii, environment and self check groups, joint-limit scale)
inside one struct per robot, usable from host C++ (the CPU oracle) and from
CUDA device code (the checker kernels), where unrolled loops over the tables
fold every offset into immediate operands.

Usage::

    python gen_header.py panda.json ../csrc/robot_panda.h
"""
import json
import math
import sys

import numpy as np

# Joint-limit scale q = u * s_m + s_a, as the reference robot structs define
# it (src/Robots.hh:17-41 Panda, :72-98 Fetch, :128-166 Baxter).
LIMITS = {
    "panda": ([5.9342, 3.6652, 5.9342, 3.2289, 5.9342, 3.9095999999999997, 5.9342],
              [-2.9671, -1.8326, -2.9671, -3.1416, -2.9671, -0.0873, -2.9671]),
    "fetch": ([0.38615, 3.2112, 2.739, 6.28318, 4.502, 6.28318, 4.32, 6.28318],
              [0.0, -1.6056, -1.221, -3.14159, -2.251, -3.14159, -2.16, -3.14159]),
    "baxter": ([3.40335987756, 3.194, 6.10835987756, 2.6679999999999997, 6.118, 3.66479632679, 6.118] * 2,
               [-1.70167993878, -2.147, -3.05417993878, -0.05, -3.059, -1.57079632679, -3.059] * 2),
}

# Arithmetic operations of one generated FK evaluation (operators plus sin/cos
# calls of the reference's straight-line FK statements): used for the
# algorithmic FLOP count.
FK_FLOPS = {"panda": 1150, "fetch": 983, "baxter": 1792}

# Rows per tile of the sample table (sphere-major inside a tile): 32 makes the FK
# kernel's stores coalesced, 1 keeps each row contiguous for the check kernel's
# bound and leaf reads.  Measured on B200: tiling speeds up the Fetch and Baxter
# checks (126 / 107 spheres per row, FP64 FK) by 5-6 % and slowed Panda's (70
# spheres at the time, a check dominated by its walk) by 6 %.
TABLE_TILE = {"panda": 1, "fetch": 32, "baxter": 32}

# Resident warps per SM the check kernel is compiled for (its register budget
# is 65536 / (32 x this)).  Swept on B200 (uneven / multi workloads, autotuned
# launch shapes): Panda 48 (40 registers) beats 40 and 56; Fetch's
# overhang-aware walk, re-swept with the certain-hit test and the shared pass
# counter, is best at 40 (48 registers: 1.85 ms against 1.90 at 32 and 2.16 at
# 24); Baxter's at 28 (72 registers: 3.12 ms against 3.13 at 32, 3.28 at 24).
CHECK_WARPS_PER_SM = {"panda": 48, "fetch": 40, "baxter": 28}


def rpy_matrix(r, p, y):
    cr, sr = math.cos(r), math.sin(r)
    cp, sp = math.cos(p), math.sin(p)
    cy, sy = math.cos(y), math.sin(y)
    rx = np.array([[1, 0, 0], [0, cr, -sr], [0, sr, cr]])
    ry = np.array([[cp, 0, sp], [0, 1, 0], [-sp, 0, cp]])
    rz = np.array([[cy, -sy, 0], [sy, cy, 0], [0, 0, 1]])
    return rz @ ry @ rx


def fmt(v):
    return repr(float(v))


def main():
    src, out = sys.argv[1], sys.argv[2]
    m = json.load(open(src))
    name = m["robot"]
    S = name.capitalize() + "Model"
    dof = m["dof"]
    sph = m["spheres"]
    env = m["env_groups"]
    slf = m["self_groups"]
    s_m, s_a = LIMITS[name]

    lines = []
    w = lines.append
    w("// Generated by batch-cc_b200/robots/gen_header.py from %s.json -- do not edit." % name)
    w("// Kinematic tree + collision-sphere tables of the %s robot, extracted from the" % name)
    w("// reference's generated fkcc<%s> (src/utils.cuh) and verified against it in FP64." % name.capitalize())
    w("#pragma once")
    w("")
    w("namespace bcc {")
    w("")
    w("struct %s {" % S)
    w("    static constexpr int dof = %d;" % dof)
    w("    static constexpr int num_spheres = %d;" % len(sph))
    w("    static constexpr int num_env_groups = %d;" % len(env))
    w("    static constexpr int num_env_leaves = %d;" % sum(len(g["leaves"]) for g in env))
    w("    static constexpr int num_self_groups = %d;" % len(slf))
    w("    static constexpr int num_self_pairs = %d;" % sum(len(g["pairs"]) for g in slf))
    w("")
    w("    // FK arithmetic width of the reference's generated code for this robot")
    w("    // (32: float expressions; 64: double expressions, centres rounded to float).")
    w("    static constexpr int fk_precision = %d;" % m.get("fk_precision", 32))
    w("    static constexpr int fk_flops = %d;" % FK_FLOPS[name])
    w("    // Sample-table rows per tile (sphere-major inside a tile; 1 = row-major).")
    w("    static constexpr int table_tile = %d;" % TABLE_TILE[name])
    w("    // Resident warps per SM the check kernel is compiled for (register budget).")
    w("    static constexpr int check_warps_per_sm = %d;" % CHECK_WARPS_PER_SM[name])
    w("")
    w("    // Fixed transform of joint k (row-major 3x4: rotation | translation).")
    w("    // frame k+1 = frame joint_parent[k] * F_k * J_k(q_k), J = Rz(q) for a revolute")
    w("    // joint (type 0), Tz(q) for a prismatic one (type 1); frame 0 is the base.")
    w("    static constexpr double joint_tf[%d][12] = {" % dof)
    parents, types = [], []
    for k, j in enumerate(m["joints"]):
        if "tf" in j:
            vals = j["tf"]
        else:
            R = rpy_matrix(*j["rpy"])
            t = j["xyz"]
            vals = [R[0, 0], R[0, 1], R[0, 2], t[0], R[1, 0], R[1, 1], R[1, 2], t[1],
                    R[2, 0], R[2, 1], R[2, 2], t[2]]
        parents.append(j.get("parent_frame", k))
        types.append(1 if j.get("type") == "prismatic" else 0)
        w("        {%s}," % ", ".join(fmt(v) for v in vals))
    w("    };")
    w("    static constexpr int joint_parent[%d] = {%s};" % (dof, ", ".join(map(str, parents))))
    w("    static constexpr int joint_type[%d] = {%s};" % (dof, ", ".join(map(str, types))))
    w("")
    w("    // Sphere k: chain frame (0 = base), offset in that frame (m), radius (m, float).")
    w("    static constexpr int sphere_frame[%d] = {%s};" % (
        len(sph), ", ".join(str(s["frame"]) for s in sph)))
    w("    static constexpr double sphere_local[%d][3] = {" % len(sph))
    for s in sph:
        w("        {%s}," % ", ".join(fmt(v) for v in s["local"]))
    w("    };")
    w("    static constexpr float sphere_radius[%d] = {%s};" % (
        len(sph), ", ".join(repr(float(np.float32(s["r"]))) + "f" for s in sph)))
    w("")
    w("    // The checker's environment groups: group g gates on sphere env_bound[g] and")
    w("    // then tests leaves env_leaves[env_leaf_begin[g] .. env_leaf_begin[g+1]).")
    w("    static constexpr int env_bound[%d] = {%s};" % (len(env), ", ".join(str(g["bound"]) for g in env)))
    begins = [0]
    for g in env:
        begins.append(begins[-1] + len(g["leaves"]))
    w("    static constexpr int env_leaf_begin[%d] = {%s};" % (len(begins), ", ".join(map(str, begins))))
    w("    static constexpr int env_leaves[%d] = {%s};" % (
        begins[-1], ", ".join(str(i) for g in env for i in g["leaves"])))
    w("    // Leaves of group g that may stick out of its bound (the first env_over_count[g]")
    w("    // of the group's leaves) and the radius (m) the bound must grow by to contain")
    w("    // every leaf at any joint value; 0 where all leaves lie inside the bound.")
    w("    static constexpr int env_over_count[%d] = {%s};" % (
        len(env), ", ".join(str(g.get("over_count", 0)) for g in env)))
    w("    static constexpr float env_cull_pad[%d] = {%s};" % (
        len(env), ", ".join(repr(float(np.float32(g.get("cull_pad", 0.0)))) + "f" for g in env)))
    w("")
    ref = m.get("ref_env_groups", env)
    w("    // The reference's own environment groups (the oracle walks these); equal to")
    w("    // the groups above where the checker keeps the reference's grouping.")
    w("    static constexpr int num_ref_env_groups = %d;" % len(ref))
    w("    static constexpr int ref_env_bound[%d] = {%s};" % (len(ref), ", ".join(str(g["bound"]) for g in ref)))
    rb = [0]
    for g in ref:
        rb.append(rb[-1] + len(g["leaves"]))
    w("    static constexpr int ref_env_leaf_begin[%d] = {%s};" % (len(rb), ", ".join(map(str, rb))))
    w("    static constexpr int ref_env_leaves[%d] = {%s};" % (
        rb[-1], ", ".join(str(i) for g in ref for i in g["leaves"])))
    w("")
    w("    // Self checks in reference order: group g gates on the bound pair self_bound[g]")
    w("    // and then tests the leaf pairs self_pairs[self_pair_begin[g] .. self_pair_begin[g+1]).")
    w("    static constexpr int self_bound[%d][2] = {%s};" % (
        len(slf), ", ".join("{%d, %d}" % tuple(g["bound"]) for g in slf)))
    pb = [0]
    for g in slf:
        pb.append(pb[-1] + len(g["pairs"]))
    w("    static constexpr int self_pair_begin[%d] = {%s};" % (len(pb), ", ".join(map(str, pb))))
    w("    static constexpr unsigned char self_pairs[%d][2] = {" % pb[-1])
    flat = ["{%d, %d}" % tuple(p) for g in slf for p in g["pairs"]]
    for i in range(0, len(flat), 12):
        w("        %s," % ", ".join(flat[i:i + 12]))
    w("    };")
    w("")
    # Sample-table row order: env-group bounds first (group order), then the
    # env-checked leaves in env_leaves order, then every other sphere.
    order = [g["bound"] for g in env] + [i for g in env for i in g["leaves"]]
    order += [i for i in range(len(sph)) if i not in order]
    assert len(set(order)) == len(order) == len(sph), "a sphere holds two table roles"
    pos = [0] * len(sph)
    for k, i in enumerate(order):
        pos[i] = k
    w("    // Position of sphere k in a sample-table row: the env-group bounding spheres")
    w("    // first (group order), then the env-checked leaves (env_leaves order), then")
    w("    // the rest; so a sample's bounds are contiguous and leaf j sits at groups + j.")
    w("    static constexpr int table_pos[%d] = {%s};" % (len(sph), ", ".join(map(str, pos))))
    w("")
    w("    // Joint-limit scale of the robot description: q = u * s_m + s_a.")
    w("    static constexpr float s_m[%d] = {%s};" % (dof, ", ".join(repr(float(np.float32(v))) + "f" for v in s_m)))
    w("    static constexpr float s_a[%d] = {%s};" % (dof, ", ".join(repr(float(np.float32(v))) + "f" for v in s_a)))
    w("};")
    w("")
    w("}  // namespace bcc")
    w("")
    open(out, "w").write("\n".join(lines))
    print("wrote", out)


if __name__ == "__main__":
    main()
