"""Robot-model extractor: generated reference FK+CC code -> kinematic tables.

The reference ships, per robot, one generated straight-line device function
``fkcc<Robot>`` (``src/utils.cuh:342-5443`` for Panda).  It evaluates the
forward kinematics of every collision sphere with scalar expressions and then
runs a fixed hierarchy of tests:

* environment checks (``src/utils.cuh:806-1190``): per link, a bounding
  sphere gate followed by that link's leaf spheres; ``panda_link0`` is
  commented out and never checked;
* self checks (``src/utils.cuh:1192-5440``): per link pair, a bounding
  sphere pair gate followed by the leaf-sphere pairs.

This script reads that function as TEXT, evaluates its FK expressions in FP64
with numpy, and re-expresses the robot as data of this project's own format:

* a serial chain of revolute joints about local z (fixed transform per joint);
* every sphere as (frame index, local offset, radius);
* the gate/leaf structure of the environment and self checks, in the
  reference's order.

For Panda the chain parameters are the public Franka Panda joint origins; the
script verifies that the chain reproduces every sphere centre of the generated
code to FP64 rounding over random configurations before writing anything.

Fetch (``fkcc<Fetch>``, ``src/utils.cuh:10382-24992``) and Baxter
(``fkcc<Baxter>``, ``:24994-38241``) are generated in a different style (SSA
``auto NAME = EXPR;`` statements, FK interleaved with the checks); for them
the kinematic tree (revolute and prismatic joints, two arms for Baxter) is
fitted to the evaluated expressions by ``fit_tree.py`` and verified the same
way.  Baxter's generated FK composes quaternions whose constants carry seven
digits (0.7071068, 0.9238792, ...), so it is rigid only to about 2e-7 m; the
fitted tree reproduces it to that level.

Usage (reads the reference tree; run in the development container only)::

    python extract_robot.py <path-to-reference>/src/utils.cuh panda panda.json [golden.json]
    python extract_robot.py <path-to-reference>/src/utils.cuh fetch fetch.json [golden.json]
"""
import json
import math
import re
import sys

import numpy as np

# cos/sin of the rounded right angle used by the robot description the
# generated code was produced from (its FK carries cos(1.57079632679) =
# 4.89663865010925e-12 wherever a joint frame is rotated by +-90 degrees).
HALF_PI_DESC = 1.57079632679

# Franka Panda joint origins (xyz, rpy) of joints 1..7; each joint rotates
# about its local z axis.  Public robot description values.
PANDA_JOINTS = [
    ((0.0, 0.0, 0.333), (0.0, 0.0, 0.0)),
    ((0.0, 0.0, 0.0), (-HALF_PI_DESC, 0.0, 0.0)),
    ((0.0, -0.316, 0.0), (HALF_PI_DESC, 0.0, 0.0)),
    ((0.0825, 0.0, 0.0), (HALF_PI_DESC, 0.0, 0.0)),
    ((-0.0825, 0.384, 0.0), (-HALF_PI_DESC, 0.0, 0.0)),
    ((0.0, 0.0, 0.0), (HALF_PI_DESC, 0.0, 0.0)),
    ((0.088, 0.0, 0.0), (HALF_PI_DESC, 0.0, 0.0)),
]

# link name -> chain frame the link is rigidly attached to (0 = base).
PANDA_LINK_FRAME = {
    "panda_link0": 0, "panda_link1": 1, "panda_link2": 2, "panda_link3": 3,
    "panda_link4": 4, "panda_link5": 5, "panda_link6": 6, "panda_link7": 7,
    "panda_hand": 7, "panda_leftfinger": 7, "panda_rightfinger": 7,
}


def rpy_matrix(r, p, y):
    cr, sr = math.cos(r), math.sin(r)
    cp, sp = math.cos(p), math.sin(p)
    cy, sy = math.cos(y), math.sin(y)
    rx = np.array([[1, 0, 0], [0, cr, -sr], [0, sr, cr]])
    ry = np.array([[cp, 0, sp], [0, 1, 0], [-sp, 0, cp]])
    rz = np.array([[cy, -sy, 0], [sy, cy, 0], [0, 0, 1]])
    return rz @ ry @ rx


def fixed_tf(xyz, rpy):
    t = np.eye(4)
    t[:3, :3] = rpy_matrix(*rpy)
    t[:3, 3] = xyz
    return t


def rot_z(q):
    c, s = math.cos(q), math.sin(q)
    t = np.eye(4)
    t[0, 0], t[0, 1], t[1, 0], t[1, 1] = c, -s, s, c
    return t


def chain_frames(joints, q):
    """World transforms of frames 0..len(joints) for configuration q (FP64)."""
    frames = [np.eye(4)]
    for (xyz, rpy), qj in zip(joints, q):
        frames.append(frames[-1] @ fixed_tf(xyz, rpy) @ rot_z(qj))
    return frames


def _function_body(text, robot_struct):
    m = re.search(r"fkcc<ppln::robots::%s>\(volatile float \*(\w+)" % robot_struct, text)
    if not m:
        raise SystemExit("fkcc<%s> not found" % robot_struct)
    start = text.index("{", m.end())
    depth, i = 0, start
    while True:
        c = text[i]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return m.group(1), text[start + 1:i]
        i += 1


def _strip_line_comment(line):
    k = line.find("//")
    return line if k < 0 else line[:k]


def parse_panda_style(body):
    """Split a Panda-style generated body into FK statements and checks."""
    lines = body.split("\n")
    # FK: everything before the first environment check.
    first_if = next(i for i, l in enumerate(lines) if "sphere_environment_in_collision" in l)
    fk_text = "\n".join(_strip_line_comment(l) for l in lines[:first_if])
    fk_text = fk_text.rsplit("if", 1)[0] if fk_text.rstrip().endswith("(") else fk_text
    stmts = []
    for s in fk_text.split(";"):
        s = " ".join(s.split())
        if not s:
            continue
        s = re.sub(r"^float\s+", "", s)
        name, expr = s.split("=", 1)
        stmts.append((name.strip(), expr.strip()))

    # Checks: walk lines after the FK, track brace depth and link comments.
    env_groups, self_groups = [], []
    depth = 0
    cur_link = None
    pending = None  # accumulates a multi-line call
    call_re_env = re.compile(r"sphere_environment_in_collision\(\s*environment\s*,([^)]*)\)")
    call_re_self = re.compile(r"sphere_sphere_self_collision\(([^)]*)\)")
    for raw in lines[first_if - 3:]:
        cm = re.match(r"\s*//\s*(panda_\w+)(?:\s+vs\.\s+(panda_\w+))?\s*$", raw)
        if cm:
            cur_link = (cm.group(1), cm.group(2))
            continue
        line = _strip_line_comment(raw)
        if pending is not None:
            pending += " " + line
        elif "sphere_environment_in_collision" in line or "sphere_sphere_self_collision" in line:
            pending = line
        if pending is not None and pending.count("(") <= pending.count(")"):
            me = call_re_env.search(pending)
            ms = call_re_self.search(pending)
            if me:
                args = [a.strip() for a in me.group(1).split(",")]
                if depth == 0:
                    env_groups.append({"link": cur_link[0], "bound": args, "leaves": []})
                else:
                    env_groups[-1]["leaves"].append(args)
            elif ms:
                args = [a.strip() for a in ms.group(1).split(",")]
                a, b = args[:4], args[4:]
                if depth == 0:
                    self_groups.append({"links": list(cur_link), "bound": [a, b], "leaves": []})
                else:
                    self_groups[-1]["leaves"].append([a, b])
            pending = None
        depth += line.count("{") - line.count("}")
    return stmts, env_groups, self_groups


def make_evaluator(stmts, qname):
    code = []
    for name, expr in stmts:
        e = expr.replace("__sinf(", "np.sin(").replace("__cosf(", "np.cos(")
        e = re.sub(r"%s\[(\d+)\]" % qname, r"q[\1]", e)
        code.append("    %s = %s" % (name, e))
    names = sorted({n for n, _ in stmts})
    src = "def fk(q):\n" + "\n".join(code) + "\n    return {%s}\n" % ", ".join(
        "'%s': %s" % (n, n) for n in names)
    ns = {"np": np}
    exec(src, ns)  # the expressions are plain arithmetic on q
    return ns["fk"]


def extract_panda(utils_path):
    text = open(utils_path).read()
    qname, body = _function_body(text, "Panda")
    stmts, env_groups, self_groups = parse_panda_style(body)
    fk = make_evaluator(stmts, qname)
    dof = 7

    # Collect every sphere referenced by a check: (x, y, z, r) variable tuples.
    sphere_keys = []
    def key_of(args):
        k = tuple(args)
        if k not in sphere_keys:
            sphere_keys.append(k)
        return sphere_keys.index(k)

    link_of = {}
    envs = []
    for g in env_groups:
        b = key_of(g["bound"])
        link_of[b] = g["link"]
        leaves = []
        for l in g["leaves"]:
            i = key_of(l)
            link_of[i] = g["link"]
            leaves.append(i)
        envs.append({"link": g["link"], "bound": b, "leaves": leaves})
    selfs = []
    for g in self_groups:
        la, lb = g["links"]
        ba, bb = key_of(g["bound"][0]), key_of(g["bound"][1])
        link_of.setdefault(ba, la)
        link_of.setdefault(bb, lb)
        pairs = []
        for a, b in g["leaves"]:
            ia, ib = key_of(a), key_of(b)
            link_of.setdefault(ia, la)
            link_of.setdefault(ib, lb)
            pairs.append([ia, ib])
        selfs.append({"links": [la, lb], "bound": [ba, bb], "pairs": pairs})

    rng = np.random.default_rng(1234)
    def value(vals, tok):
        try:
            return float(tok)
        except ValueError:
            return float(vals[tok])

    # Local offsets from q = random reference pose, then verification.
    q0 = rng.uniform(-3.0, 3.0, dof)
    vals = fk(q0)
    frames = chain_frames(PANDA_JOINTS, q0)
    spheres = []
    for idx, k in enumerate(sphere_keys):
        frame = PANDA_LINK_FRAME[link_of[idx]]
        p = np.array([value(vals, t) for t in k[:3]] + [1.0])
        local = np.linalg.solve(frames[frame], p)[:3]
        r = float(np.float32(value(vals, k[3])))
        spheres.append({"frame": frame, "local": local.tolist(), "r": r,
                        "link": link_of[idx], "src": list(k)})

    max_err = 0.0
    for _ in range(2000):
        q = rng.uniform(-4.0, 4.0, dof)
        vals = fk(q)
        frames = chain_frames(PANDA_JOINTS, q)
        for s in spheres:
            p = frames[s["frame"]] @ np.array(s["local"] + [1.0])
            ref = np.array([value(vals, t) for t in s["src"][:3]])
            max_err = max(max_err, float(np.abs(p[:3] - ref).max()))
    if max_err > 1e-12:
        raise SystemExit("chain does not reproduce the generated FK: max err %g" % max_err)

    # Leaf-in-bound containment (decides whether gates can change verdicts).
    contain = []
    for g in envs:
        b = spheres[g["bound"]]
        worst = -1e9
        for i in g["leaves"]:
            s = spheres[i]
            assert s["frame"] == b["frame"]
            d = np.linalg.norm(np.array(s["local"]) - np.array(b["local"])) + s["r"] - b["r"]
            worst = max(worst, d)
        contain.append({"link": g["link"], "leaf_excess_m": worst})
    for g in selfs:
        for side in (0, 1):
            b = spheres[g["bound"][side]]
            worst = -1e9
            for p in g["pairs"]:
                s = spheres[p[side]]
                d = np.linalg.norm(np.array(s["local"]) - np.array(b["local"])) + s["r"] - b["r"]
                worst = max(worst, d)
            contain.append({"link": g["links"][side], "pair": g["links"], "leaf_excess_m": worst})

    return {
        "robot": "panda",
        "dof": dof,
        "joints": [{"xyz": list(x), "rpy": list(r)} for x, r in PANDA_JOINTS],
        "spheres": [{k: s[k] for k in ("frame", "local", "r", "link")} for s in spheres],
        "env_groups": envs,
        "self_groups": selfs,
        "containment": contain,
        "fk_max_abs_err_vs_generated_code_m": max_err,
        "_fk_eval": fk,
        "_sphere_src": [s["src"] for s in spheres],
    }


# The checker's environment groups for Panda: its own bounding hierarchy over
# the reference's 58 leaves (the reference's groups stay in the model as
# "ref_env_groups", which the oracle walks).  Every leaf lies inside its
# group's bound, so a leaf that hits a primitive implies its bound hits it and
# any such grouping gives the reference's verdicts; the grouping only sets the
# checker's work: one bound test per (primitive, group) candidate at every
# sample walked, and the group's leaf tests after each bound hit.  Ten groups
# (one warp culls three pairs at ten lanes each), chosen per link frame with a
# cost model measured on the uneven workload -- bound and leaf tests of
# collision-free pairs over all their samples, and of colliding pairs at their
# first sample: link 7, the hand and both fingers (frame 7) under one bound,
# link 5 in two clusters, links 2 and 1 in halves, links 6, 4 and 3 under the
# reference's bound (already the smallest sphere enclosing their leaves).
# Against the reference's grouping the model predicts half the bound and leaf
# tests per sample of collision-free pairs and 18 % fewer at the first sample
# of colliding pairs (measured on the GPU: 12 % fewer candidates per pair, a
# quarter fewer leaf steps).
PANDA_CHECK_GROUPS = [
    [1, 2, 4, 5] + list(range(7, 25)) + list(range(26, 31)),  # fingers, hand, link 7
    [32, 33, 34],                                            # link 6
    [36, 37, 41, 42, 43, 45, 46, 47], [38, 39, 40, 44],      # link 5
    [49, 50, 51, 52],                                        # link 4
    [54, 55, 56, 57],                                        # link 3
    [59, 60], [61, 62],                                      # link 2
    [64, 65], [66, 67],                                      # link 1
]
CHECK_BOUND_MARGIN = 1e-5  # radius added to a new bound beyond its leaves (m), far above FP32 FK rounding


def regroup(model, partition):
    """Replace the model's environment groups by `partition` (lists of leaf
    sphere indices, each within one frame).  A list equal to a reference
    group's leaves keeps that group's bound; any other gets a new bound sphere
    (appended, "src" -1): the smallest sphere enclosing its leaves plus
    CHECK_BOUND_MARGIN, radius rounded up to float."""
    import fit_tree

    spheres = [dict(s, src=i) for i, s in enumerate(model["spheres"])]
    ref = model["env_groups"]
    ref_leaves = sorted(i for g in ref for i in g["leaves"])
    if sorted(i for p in partition for i in p) != ref_leaves:
        raise SystemExit("the check groups must hold every reference leaf exactly once")
    by_leaves = {tuple(g["leaves"]): g for g in ref}
    groups = []
    for leaves in partition:
        frames = {spheres[i]["frame"] for i in leaves}
        if len(frames) != 1:
            raise SystemExit("check group %s spans frames %s" % (leaves, sorted(frames)))
        links = "+".join(dict.fromkeys(spheres[i]["link"] for i in leaves))
        g0 = by_leaves.get(tuple(leaves))
        if g0 is not None:
            groups.append({"link": g0["link"], "bound": g0["bound"], "leaves": list(leaves)})
            continue
        c, r = fit_tree.smallest_enclosing_sphere([spheres[i]["local"] for i in leaves],
                                                   [spheres[i]["r"] for i in leaves])
        r32 = float(np.nextafter(np.float32(r + CHECK_BOUND_MARGIN), np.float32(np.inf)))
        spheres.append({"frame": frames.pop(), "local": list(map(float, c)), "r": r32, "link": links, "src": -1})
        groups.append({"link": links, "bound": len(spheres) - 1, "leaves": list(leaves)})
    out = dict(model)
    out["spheres"] = spheres
    out["env_groups"] = groups
    out["ref_env_groups"] = ref
    return out


SSA_DOF = {"fetch": 8, "baxter": 14}
MAX_ENV_GROUPS = 32       # one lane per group in the checker's cull
OVERHANG_EPS = 1e-6       # leaves sticking out less than this count as contained (m)
CULL_PAD_MARGIN = 1e-5    # extra cull radius on top of the measured overhang (m)


def extract_ssa(utils_path, robot):
    """Fetch / Baxter: generated SSA code -> fitted kinematic tree + tables.

    Check groups keep the reference's bound/leaf structure with three
    adjustments the checker's table layout needs (none changes a verdict):
    a group without leaves tests its bound sphere directly, so it gets that
    sphere as its one leaf; a sphere used in several roles (bound of one
    group, leaf of another) is duplicated so that every role has its own
    sample-table row; and when there are more than 32 groups, leafless
    groups on the same frame are merged under a synthetic bound that encloses
    them (a leaf inside its bound needs no gate of its own)."""
    import fit_tree

    text = open(utils_path).read()
    qname, body = _function_body(text, robot.capitalize())
    stmts, env_raw, self_raw = fit_tree.parse_ssa(body)
    dof = SSA_DOF[robot]
    keys = []

    def key(t):
        if t not in keys:
            keys.append(t)
        return keys.index(t)

    for g in env_raw:
        key(g["bound"])
        for l in g["leaves"]:
            key(l)
    for g in self_raw:
        key(g["bound"][0])
        key(g["bound"][1])
        for a, b in g["pairs"]:
            key(a)
            key(b)
    fk = fit_tree.make_evaluator(stmts, qname)
    rng = np.random.default_rng(1234)
    joints, body_of, base = fit_tree.fit_tree(fk, keys, dof, rng)
    mj, frames, local = fit_tree.to_model(joints, body_of, base)

    max_err = 0.0
    for _ in range(2000):
        q = rng.uniform(-4.0, 4.0, dof)
        want = fit_tree.centres(fk, keys, q[None])[:, 0, :]
        got = fit_tree.chain_centres(mj, frames, local, q)
        max_err = max(max_err, float(np.abs(got - want).max()))
    if max_err > 1e-6:
        raise SystemExit("fitted tree does not reproduce the generated FK: max err %g" % max_err)

    spheres = [{"frame": frames[i], "local": list(map(float, local[i])), "r": float(np.float32(float(k[3]))),
                "link": None, "src": i} for i, k in enumerate(keys)]
    used = set()

    def role(i):
        """Sphere index for a new table role of source sphere i (duplicated if taken)."""
        if i not in used:
            used.add(i)
            return i
        spheres.append(dict(spheres[i]))
        return len(spheres) - 1

    groups = [{"link": g["link"] or "unnamed", "bound": key(g["bound"]),
               "leaves": [key(l) for l in g["leaves"]]} for g in env_raw]
    if len(groups) > MAX_ENV_GROUPS:
        by_frame = {}
        for gi, g in enumerate(groups):
            if not g["leaves"]:
                by_frame.setdefault(frames[g["bound"]], []).append(gi)
        merged, drop = [], set()
        for f, gis in sorted(by_frame.items()):
            if len(gis) < 2 or len(groups) - len(drop) <= MAX_ENV_GROUPS:
                continue
            mem = [groups[gi]["bound"] for gi in gis]
            c, r = fit_tree.enclosing_sphere([local[m] for m in mem], [spheres[m]["r"] for m in mem])
            r32 = float(np.nextafter(np.float32(r + 1e-6), np.float32(np.inf)))
            spheres.append({"frame": f, "local": list(map(float, c)), "r": r32, "link": None, "src": -1})
            merged.append({"link": "+".join(groups[gi]["link"] for gi in gis), "bound": len(spheres) - 1,
                           "leaves": mem, "synthetic": True})
            drop.update(gis)
        groups = [g for gi, g in enumerate(groups) if gi not in drop] + merged
    if len(groups) > MAX_ENV_GROUPS:
        raise SystemExit("%d environment groups (max %d)" % (len(groups), MAX_ENV_GROUPS))

    envs = []
    for g in groups:
        b_src = g["bound"]
        leaves_src = g["leaves"] if g["leaves"] else [b_src]
        b = role(b_src) if not g.get("synthetic") else b_src
        # overhang of each leaf beyond the bound, max over all joint values
        over = []
        for l in leaves_src:
            d = fit_tree.max_distance(mj, spheres[l]["frame"], np.array(spheres[l]["local"]),
                                      spheres[b]["frame"], np.array(spheres[b]["local"]), dof)
            over.append(d + spheres[l]["r"] - spheres[b]["r"])
        order = sorted(range(len(leaves_src)), key=lambda i: (over[i] <= OVERHANG_EPS, i))
        leaves = [role(leaves_src[i]) for i in order]
        n_over = sum(1 for o in over if o > OVERHANG_EPS)
        pad = max([0.0] + [o for o in over if o > OVERHANG_EPS])
        pad = float(np.float32(pad + CULL_PAD_MARGIN)) if n_over else 0.0
        for i in [b] + leaves:
            spheres[i]["link"] = spheres[i]["link"] or g["link"]
        envs.append({"link": g["link"], "bound": b, "leaves": leaves, "over_count": n_over, "cull_pad": pad,
                     "max_overhang_m": max(over)})
    selfs = []
    for g in self_raw:
        la, lb = g["links"] if g["links"] else ("?", "?")
        pairs = [[key(a), key(b)] for a, b in g["pairs"]]
        ba, bb = key(g["bound"][0]), key(g["bound"][1])
        if not pairs:
            pairs = [[ba, bb]]
        selfs.append({"links": [la, lb], "bound": [ba, bb], "pairs": pairs})
    for s in spheres:
        s["link"] = s["link"] or "self_only"
    return {
        "robot": robot,
        "dof": dof,
        "fk_precision": 64,
        "joints": mj,
        "spheres": [{k: s[k] for k in ("frame", "local", "r", "link", "src")} for s in spheres],
        "env_groups": envs,
        "self_groups": selfs,
        "fk_max_abs_err_vs_generated_code_m": max_err,
        "_fk_eval": fk,
        "_sphere_src": keys,
    }


def main():
    utils_path, robot, out = sys.argv[1], sys.argv[2], sys.argv[3]
    model = regroup(extract_panda(utils_path), PANDA_CHECK_GROUPS) if robot == "panda" else \
        extract_ssa(utils_path, robot)
    fk = model.pop("_fk_eval")
    src = model.pop("_sphere_src")
    # Golden FK vectors: sphere centres of the generated code (FP64) at seeded q.
    rng = np.random.default_rng(20261203)
    gold = []
    for _ in range(64):
        q = rng.uniform(-3.2, 3.9, model["dof"]).astype(np.float32).astype(np.float64)
        vals = fk(q) if robot == "panda" else {k: v[0] for k, v in fk(q[None]).items() if k != "q"}
        cs = []
        for k in src:
            cs.append([float(vals[t]) if not re.match(r"^-?[\d.]", t) else float(t) for t in k[:3]])
        gold.append({"q": q.tolist(), "centres": cs})
    gold_doc = {"robot": robot, "cases": gold}
    # model sphere -> index into "centres" (-1: synthetic bound, no source)
    gold_doc["src_of_sphere"] = [s["src"] for s in model["spheres"]]
    with open(out, "w") as f:
        json.dump(model, f, indent=1)
    if len(sys.argv) > 4:
        with open(sys.argv[4], "w") as f:
            json.dump(gold_doc, f)
    print("spheres=%d env_groups=%d self_groups=%d self_pairs=%d fk_err=%.3g" % (
        len(model["spheres"]), len(model["env_groups"]), len(model["self_groups"]),
        sum(len(g["pairs"]) for g in model["self_groups"]),
        model["fk_max_abs_err_vs_generated_code_m"]))
    for c in model.get("containment", []):
        if c["leaf_excess_m"] > 0:
            print("leaf outside bound:", c)
    for g in model["env_groups"]:
        if g.get("over_count"):
            print("group %s: %d leaves overhang the bound by up to %.3g m" % (g["link"], g["over_count"],
                                                                              g["max_overhang_m"]))


if __name__ == "__main__":
    main()
