"""Hand-built known-answer cases shared by the CPU and GPU tests."""
import json
import os

import numpy as np

from bcc import EnvSet, workload
from bcc.workload import make_spheres
from oracle import oracle as orc

ROBOTS_DIR = os.path.join(os.path.dirname(__file__), "..", "batch-cc_b200", "robots")
INFLATE = 0.005


def robot_model(robot):
    with open(os.path.join(ROBOTS_DIR, robot + ".json")) as f:
        return json.load(f)


def overhang_case(robot, seed=0):
    """A configuration q and three one- or two-sphere environments that separate
    the reference's gate semantics from per-primitive gating.

    A leaf l of some group sticks out of the group's bound b by o > 0.1 mm at
    q.  Obstacle A lies in that overhang: the leaf reaches o / 2 into it, the
    bound stays o / 2 short, and no other robot sphere reaches it.  Obstacle B
    dents the bound by 1 mm in a direction away from every leaf of the group.
    Reference semantics (leaves are tested only after the bound hit some
    primitive): {A} free, {B} free, {A, B} colliding -- while a checker gating
    each leaf on the bound hitting the SAME primitive would call {A, B} free.
    Returns (q, EnvSet [{A}, {B}, {A, B}], expected verdicts)."""
    m = robot_model(robot)
    r = np.array([s["r"] for s in m["spheres"]])
    groups = sorted((g for g in m["env_groups"] if g.get("over_count", 0) > 0),
                    key=lambda g: -g.get("max_overhang_m", 0.0))
    assert groups
    s_m, s_a = workload.LIMITS[robot]
    rng = np.random.default_rng(seed)
    empty = EnvSet.from_lists([{}])
    ra = 0.005
    for _ in range(400):
        q = (rng.uniform(0, 1, len(s_m)) * s_m + s_a).astype(np.float32)
        if orc.config_collides(empty, 0, q, robot=robot):
            continue  # self-collision
        c = orc.fk(q, robot)
        for g in groups:
            b = g["bound"]
            leaves = np.array(g["leaves"])
            for l in g["leaves"][:g["over_count"]]:
                o = np.linalg.norm(c[l] - c[b]) + r[l] - r[b]
                if o < 1e-4:
                    continue
                u = (c[l] - c[b]) / np.linalg.norm(c[l] - c[b])
                ca = c[b] + u * (r[b] + INFLATE + o / 2 + ra)
                # B: the direction on the bound farthest from every leaf of the group
                dirs = rng.normal(size=(2000, 3))
                dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
                pts = c[b] + dirs * r[b]
                gap = np.min(np.linalg.norm(pts[:, None, :] - c[leaves][None], axis=2) - r[leaves][None], axis=1)
                if gap.max() < 0.006:
                    continue
                v = dirs[np.argmax(gap)]
                cb = c[b] + v * (r[b] + INFLATE + ra - 1e-3)
                envs = EnvSet.from_lists([{"spheres": make_spheres(ca[None], [ra])},
                                          {"spheres": make_spheres(cb[None], [ra])},
                                          {"spheres": make_spheres(np.stack([ca, cb]), [ra, ra])}])
                want = [orc.config_collides(envs, i, q, robot=robot) for i in range(3)]
                if want == [False, False, True]:
                    return q, envs, np.array(want, np.uint8)
    raise RuntimeError("no overhang case found for %s" % robot)
