"""CPU tests of the oracle: pinned to the reference's generated FK, the
reference discretisation rules, and hand-built known-answer cases."""
import json
import os

import numpy as np
import pytest

from bcc import EnvSet, workload
from bcc.workload import make_capsules, make_cuboids, make_spheres
from oracle import oracle as orc

import cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# Largest difference between the tables' FK and the reference's generated FK
# expressions: FP64 rounding for Panda and Fetch; Baxter's generated FK
# multiplies quaternions whose constants carry 7 digits, so it is rigid only to
# about 2e-7 m and the fitted tree matches it to that level.
FK_TOL = {"panda": 1e-12, "fetch": 1e-12, "baxter": 5e-7}


@pytest.mark.parametrize("robot", ["panda", "fetch", "baxter"])
def test_fk_matches_reference_generated_code(robot):
    """Sphere centres of the robot tables == the reference's generated fkcc<Robot>
    FK expressions evaluated in FP64 (tests/golden/<robot>_fk_generated.json)."""
    g = json.load(open(os.path.join(GOLDEN, robot + "_fk_generated.json")))
    assert len(g["cases"]) >= 32
    src = g.get("src_of_sphere")
    worst = 0.0
    for c in g["cases"]:
        q = np.array(c["q"], np.float32)
        assert np.array_equal(q.astype(np.float64), np.array(c["q"]))
        got = orc.fk(q, robot)
        want = np.array(c["centres"])
        if src is None:
            worst = max(worst, float(np.abs(got - want).max()))
        else:
            idx = np.array(src)
            has = idx >= 0  # synthetic bounds have no generated counterpart
            assert sorted(set(idx[has].tolist())) == list(range(len(want)))
            worst = max(worst, float(np.abs(got[has] - want[idx[has]]).max()))
    assert worst < FK_TOL[robot], worst


@pytest.mark.parametrize("robot", ["panda", "fetch", "baxter"])
def test_leaves_stay_inside_the_padded_bound(robot):
    """Every environment leaf lies inside its group's bound grown by the group's
    cull pad, at any configuration (the checker culls with the padded bound),
    and a leaf outside the plain bound is one of the group's listed
    overhanging leaves.  Leaves within 1 um of the bound count as inside
    (Panda's stick out by 4.4e-9 m; the cull adds a 1e-4 m margin)."""
    m = cases.robot_model(robot)
    r = np.array([s["r"] for s in m["spheres"]])
    rng = np.random.default_rng(17)
    s_m, s_a = workload.LIMITS[robot]
    for _ in range(300):
        q = (rng.uniform(-0.2, 1.2, len(s_m)) * s_m + s_a).astype(np.float32)
        c = orc.fk(q, robot)
        for g in m["env_groups"]:
            b = g["bound"]
            pad = g.get("cull_pad", 0.0)
            for i, l in enumerate(g["leaves"]):
                out = np.linalg.norm(c[l] - c[b]) + r[l] - r[b]
                assert out <= pad + 1e-6, (g["link"], l, out, pad)
                if out > 1e-6:
                    assert i < g.get("over_count", 0), (g["link"], l, out)


@pytest.mark.parametrize("robot", ["fetch", "baxter"])
def test_overhang_case_separates_gate_semantics(robot):
    """The overhang known answer: the reference's semantics (oracle) give
    {A} free, {B} free, {A, B} colliding, and gating each leaf on its bound
    hitting the same primitive would call {A, B} free."""
    q, envs, want = cases.overhang_case(robot)
    assert want.tolist() == [0, 0, 1]
    v = orc.check(envs, np.stack([q, q])[None], robot=robot)
    assert v[0].tolist() == [0, 0, 1]
    # per-primitive gating on {A, B}
    m = cases.robot_model(robot)
    r = np.array([s["r"] for s in m["spheres"]]) + cases.INFLATE
    c = orc.fk(q, robot)
    obst = envs.env(2)["spheres"]  # the {A, B} environment's two spheres
    assert len(obst) == 2
    hit = lambda i, o: np.linalg.norm(c[i] - o[:3]) < r[i] + o[3]
    per_prim = any(hit(g["bound"], o) and any(hit(l, o) for l in g["leaves"])
                   for g in m["env_groups"] for o in obst)
    assert not per_prim


def test_discretisation_rules():
    # n = max(ceil(|e - s| / 31 * 32), 1): a zero-length edge still checks 32 samples.
    s = np.zeros(7, np.float32)
    assert orc.edge_n(s, s) == 1
    assert len(orc.edge_samples(s, s)) == 32
    e = s.copy()
    e[0] = 31.0 / 32.0  # exactly one step boundary
    assert orc.edge_n(s, e) == 1
    e[0] = np.nextafter(np.float32(31.0 / 32.0), np.float32(2))
    assert orc.edge_n(s, e) == 2
    e[0] = 12.0
    assert orc.edge_n(s, e) == int(np.ceil(12.0 / 31.0 * 32.0))


def test_sample_set_overshoots_like_reference():
    """Samples t_k = k / (31 n), k < 32 n: lane 31's first sample is the goal and
    the last sample lies past it (src/batch_cc.cu:109-129)."""
    rng = np.random.default_rng(0)
    for _ in range(50):
        s = rng.uniform(-2, 2, 7).astype(np.float32)
        e = (s + rng.uniform(-1.5, 1.5, 7)).astype(np.float32)
        n = orc.edge_n(s, e)
        S = orc.edge_samples(s, e)
        assert S.shape == (32 * n, 7)
        assert np.array_equal(S[0], s)  # k = 0 is the start, exactly
        t = np.arange(32 * n) / (31.0 * n)
        ideal = s[None, :].astype(np.float64) + t[:, None] * (e - s)[None, :].astype(np.float64)
        assert np.abs(S - ideal).max() < 1e-5
        assert np.abs(S[31 * n] - e).max() < 1e-5  # lane 31 starts at the goal


def test_bcc_edge_samples_matches_oracle():
    from bcc import lib as bcclib

    rng = np.random.default_rng(1)
    for _ in range(200):
        s = rng.uniform(-3, 3, 7).astype(np.float32)
        e = rng.uniform(-3, 3, 7).astype(np.float32)
        assert bcclib.edge_samples(s, e) == 32 * orc.edge_n(s, e)


def _pose_with_hand_sphere():
    q = np.array([0.3, -0.4, 0.2, -2.0, 0.1, 1.8, 0.5], np.float32)
    c = orc.fk(q)
    return q, c


def _tip_and_approach(c):
    """Outermost right-finger leaf (sphere 2) and the hand's approach axis
    (frame-7 z, through spheres 26 and 6): obstacles placed beyond the tip
    along it are nearest to that leaf alone."""
    d = c[6] - c[26]
    return 2, d / np.linalg.norm(d)


def test_known_answer_touching_sphere():
    """One obstacle sphere 1e-4 m outside / inside contact with the fingertip
    sphere (radius + 0.005 inflation): free / collision."""
    q, c = _pose_with_hand_sphere()
    tip, d = _tip_and_approach(c)
    r_tip = 0.012000000104308128
    r_obs = 0.05
    for gap, want in ((1e-4, 0), (-1e-4, 1)):
        centre = c[tip] + d * (r_tip + 0.005 + r_obs + gap)
        envs = EnvSet.from_lists([{"spheres": make_spheres(centre[None, :], np.array([r_obs]))}])
        edge = np.stack([q, q])[None]
        v = orc.check(envs, edge)
        pen, _ = orc.pair_pen(envs, edge, [[0, 0]])
        assert v[0, 0] == want, (gap, pen)
        assert abs(pen[0] + gap) < 2e-6


def test_empty_env_only_self_collision():
    edges = workload.gen_edges("uneven", 200, seed=5)
    empty = EnvSet.from_lists([{}, {}])
    v = orc.check(empty, edges)
    assert np.array_equal(v[:, 0], v[:, 1])
    assert 0 < v[:, 0].mean() < 0.5  # some edges self-collide, most do not


def test_zero_length_capsule_is_sphere():
    rng = np.random.default_rng(3)
    cen = rng.uniform(-0.5, 0.5, (6, 3))
    cap = make_capsules(cen, np.zeros((6, 3)), np.full(6, 0.08), np.zeros(6))
    assert np.all(np.isinf(cap[:, 7]))
    sph = make_spheres(cen, np.full(6, 0.08))
    envs = EnvSet.from_lists([{"capsules": cap}, {"spheres": sph}])
    edges = workload.gen_edges("plain", 60, seed=3)
    v = orc.check(envs, edges)
    assert np.array_equal(v[:, 0], v[:, 1])


def test_cylinders_are_never_tested():
    rng = np.random.default_rng(4)
    cyl = make_capsules(rng.uniform(-0.2, 0.2, (4, 3)), np.zeros((4, 3)), np.full(4, 0.3), np.full(4, 1.0))
    envs = EnvSet.from_lists([{"cylinders": cyl}, {}])
    edges = workload.gen_edges("plain", 40, seed=4)
    v = orc.check(envs, edges)
    assert np.array_equal(v[:, 0], v[:, 1])


@pytest.mark.parametrize("name,nenv,nedge", [("uneven", 24, 120), ("multi_fetch", 10, 60), ("multi_baxter", 8, 50)])
def test_fp32_and_fp64_oracles_agree_up_to_contact(name, nenv, nedge):
    robot = workload.robot_of(name)
    envs = workload.gen_envs(name, nenv, seed=11)
    edges = workload.gen_edges(name, nedge, seed=11)
    v64 = orc.check(envs, edges, precision=64, robot=robot)
    v32 = orc.check(envs, edges, precision=32, robot=robot)
    n, adj, bad = orc.adjudicate(envs, edges, v32, v64, robot=robot)
    assert len(bad) == 0


def test_penetration_sign_matches_verdict():
    envs = workload.gen_envs("plain", 6, seed=2)
    edges = workload.gen_edges("plain", 40, seed=2)
    v = orc.check(envs, edges)
    pairs = np.array([(e, i) for e in range(40) for i in range(6)])
    pen, _ = orc.pair_pen(envs, edges, pairs)
    verdict = v[pairs[:, 0], pairs[:, 1]]
    assert np.all(pen[verdict == 1] > -1e-9)
    assert np.all(pen[verdict == 0] < 1e-9)


def test_known_answer_rotated_cuboid_face():
    """A rotated cuboid whose face lies 1e-4 m outside / inside the inflated
    fingertip sphere: free / collision."""
    q, c = _pose_with_hand_sphere()
    tip, d = _tip_and_approach(c)
    r_inf = 0.012000000104308128 + 0.005
    u = np.cross(d, [0.3, 0.5, 0.8])
    u /= np.linalg.norm(u)
    w = np.cross(d, u)
    h = np.array([0.04, 0.05, 0.03])
    for gap, want in ((1e-4, 0), (-1e-4, 1)):
        centre = c[tip] + d * (r_inf + gap + h[0])
        rec = np.zeros((1, 15), np.float32)
        rec[0, 0:3] = centre
        rec[0, 3:6], rec[0, 6:9], rec[0, 9:12] = d, u, w
        rec[0, 12:15] = h
        envs = EnvSet.from_lists([{"cuboids": rec}])
        edge = np.stack([q, q])[None]
        assert orc.check(envs, edge)[0, 0] == want


LEAVES = [1, 2, 4, 5] + list(range(7, 25)) + list(range(26, 31)) + [32, 33, 34] + list(range(36, 48)) + \
    [49, 50, 51, 52, 54, 55, 56, 57, 59, 60, 61, 62, 64, 65, 66, 67]


def orc_radii():
    m = json.load(open(os.path.join(os.path.dirname(__file__), "..", "batch-cc_b200", "robots", "panda.json")))
    return np.array([s["r"] for s in m["spheres"]])


def test_leaf_list_matches_model():
    m = json.load(open(os.path.join(os.path.dirname(__file__), "..", "batch-cc_b200", "robots", "panda.json")))
    leaves = sorted(i for g in m["env_groups"] for i in g["leaves"])
    assert leaves == sorted(LEAVES)


@pytest.mark.parametrize("name", ["plain", "uneven", "stress", "multi_fetch", "multi_baxter"])
def test_workload_generators_are_seeded(name):
    a = workload.gen_envs(name, 5, seed=9)
    b = workload.gen_envs(name, 5, seed=9)
    for k in a.records:
        assert np.array_equal(a.records[k], b.records[k])
    e1 = workload.gen_edges(name, 50, seed=9)
    e2 = workload.gen_edges(name, 50, seed=9)
    assert np.array_equal(e1, e2)
    s_m, s_a = workload.LIMITS[workload.robot_of(name)]
    assert e1.shape[2] == len(s_m)
    assert np.all(e1 >= s_a - 1e-5) and np.all(e1 <= s_a + s_m + 1e-5)


def test_ordering_can_save_little_on_the_uneven_workload():
    """The workload property behind the learned-order result: with exact
    per-sample verdicts (oracle), a PERFECT ordering -- the first colliding
    sample checked first -- saves under 15 % of the plain order's sample-rank
    work on the uneven workload, because almost every colliding pair already
    collides at rank 0 (the edge's start) and collision-free pairs, which need
    every sample in any order, hold most of the work."""
    envs = workload.gen_envs("uneven", 100, seed=0)
    edges = workload.gen_edges("uneven", 1000, seed=0)
    rng = np.random.default_rng(3)
    plain = perfect = 0.0
    rank0 = colliding = 0
    for _ in range(150):
        e, v = int(rng.integers(len(edges))), int(rng.integers(envs.num_envs))
        S = orc.edge_samples(edges[e, 0], edges[e, 1])
        n = len(S) // 32
        hits = [k for k in range(len(S)) if orc.config_collides(envs, v, S[k])]
        if hits:
            r = min((k % n) * 32 + k // n for k in hits)  # reference rank of sample k = lane * n + round
            plain, perfect, colliding, rank0 = plain + r + 1, perfect + 1, colliding + 1, rank0 + (r == 0)
        else:
            plain, perfect = plain + 32 * n, perfect + 32 * n
    assert colliding > 100 and rank0 / colliding > 0.9
    assert 1.0 - perfect / plain < 0.15


def _ranks_walked(hits, n, pi):
    """Ranks a walk visits per pair when rank r checks sample pi[r % 32] * n + r // 32
    (pi = identity is the reference order, src/batch_cc.cu:118-129): up to and
    including the first colliding one, or all 32 n for a collision-free pair."""
    r = np.arange(32 * n)
    h = hits[:, pi[r % 32] * n + r // 32]
    return np.where(h.any(1), np.argmax(h, 1) + 1, 32 * n)


def test_per_edge_order_ceiling_on_the_uneven_workload():
    """What any scorer of an edge's 32 lane blocks can gain over a random block
    order (block 0 first) on the uneven workload: the exact per-sample verdicts
    of 100 000 (edge, env) pairs give, per edge, the greedy block order built
    from the answers themselves (an upper bound for a scorer that sees only the
    edge, as the one-cluster learned order does).  It beats the random order by
    a few percent of the walked ranks, while the random order already takes most
    of the per-pair perfect order's saving: the structure of the order matters
    more than the scores on this workload."""
    E, N = 1000, 100
    envs = workload.gen_envs("uneven", N, seed=0)
    edges = workload.gen_edges("uneven", E, seed=0)
    pairs = np.array([(e, v) for e in range(E) for v in range(N)], np.int64)
    S = orc.pair_samples(envs, edges, pairs) == 1
    ns = np.array([orc.edge_n(edges[e, 0], edges[e, 1], 32) for e in range(E)])
    rng = np.random.default_rng(0)
    tot = {"plain": 0, "random": 0, "reverse": 0, "per_edge_best": 0, "per_pair_perfect": 0}
    for e in range(E):
        n, h = int(ns[e]), S[e * N:(e + 1) * N]
        tot["plain"] += _ranks_walked(h, n, np.arange(32)).sum()
        tot["random"] += _ranks_walked(h, n, np.concatenate([[0], 1 + rng.permutation(31)])).sum()
        tot["reverse"] += _ranks_walked(h, n, np.concatenate([[0], np.arange(31, 0, -1)])).sum()
        alive, order, rest = ~h[:, 0], [0], list(range(1, 32))
        while rest:  # greedy: the block whose first sample decides most undecided pairs
            b = max(rest, key=lambda b: (h[alive, b * n].sum(), -b))
            order.append(b); rest.remove(b); alive &= ~h[:, b * n]
        tot["per_edge_best"] += _ranks_walked(h, n, np.array(order)).sum()
        tot["per_pair_perfect"] += np.where(h.any(1), 1, 32 * n).sum()
    save = {k: 1.0 - v / tot["plain"] for k, v in tot.items()}
    assert 0 < save["random"] < save["per_edge_best"] <= save["per_pair_perfect"] < 0.15
    assert save["per_edge_best"] - save["random"] < 0.04
    assert save["random"] > 0.6 * save["per_pair_perfect"]
