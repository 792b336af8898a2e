"""CPU tests of the checker's environment groups and of the certain-hit test.

The checker may walk its own grouping of a robot's leaves (Panda) as long as
every leaf lies inside its group's bound; the oracle walks the reference's
groups (`ref_env_groups`).  A bound whose centre lies within rho + kappa_g of a
primitive's core proves a leaf hit (bcc_pipeline.cuh `cert_radius`); the test
below restates kappa_g and checks that claim on random rounded boxes.
"""
import os
import re

import numpy as np
import pytest

import cases

HEADERS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "batch-cc_b200", "csrc")
INFLATE = 0.005          # robot sphere inflation (src/utils.cuh:215)
CERT_MARGIN = 1e-4       # margin the certain-hit radius keeps below the leaf reach


def ref_groups(m):
    return m.get("ref_env_groups", m["env_groups"])


@pytest.mark.parametrize("robot", ["panda", "fetch", "baxter"])
def test_check_groups_hold_every_reference_leaf_once(robot):
    m = cases.robot_model(robot)
    got = sorted(l for g in m["env_groups"] for l in g["leaves"])
    want = sorted(l for g in ref_groups(m) for l in g["leaves"])
    assert got == want
    assert len(got) == len(set(got))


def test_panda_check_groups_stay_in_one_frame_and_keep_ten_lanes():
    m = cases.robot_model("panda")
    sph = m["spheres"]
    assert len(m["env_groups"]) == 10          # three pairs per 32-lane cull pass
    assert len(m["ref_env_groups"]) == 10
    for g in m["env_groups"]:
        frames = {sph[i]["frame"] for i in [g["bound"]] + g["leaves"]}
        assert len(frames) == 1, g
    # the appended bounds have no counterpart in the reference's generated code
    for i, s in enumerate(sph):
        assert s["src"] == (i if i < 70 else -1)


@pytest.mark.parametrize("robot", ["panda", "fetch", "baxter"])
def test_header_carries_the_reference_groups_for_the_oracle(robot):
    """robot_<name>.h's ref_env_* tables are the JSON's reference groups."""
    m = cases.robot_model(robot)
    text = open(os.path.join(HEADERS, "robot_%s.h" % robot)).read()

    def arr(name):
        body = re.search(r"static constexpr int %s\[\d+\] = \{([^}]*)\};" % name, text).group(1)
        return [int(v) for v in body.split(",")]

    ref = ref_groups(m)
    assert arr("ref_env_bound") == [g["bound"] for g in ref]
    assert arr("ref_env_leaves") == [l for g in ref for l in g["leaves"]]
    assert arr("env_bound") == [g["bound"] for g in m["env_groups"]]


def cert_radius(m, g):
    """Restatement of cert_radius (bcc_pipeline.cuh): max over the leaves rigid
    with the bound and no larger than it of r_l + inflate - |c_l - c_b|, less
    the margin, at least 0."""
    sph = m["spheres"]
    b = sph[g["bound"]]
    best = 0.0
    for l in g["leaves"]:
        s = sph[l]
        if s["frame"] != b["frame"] or np.float32(s["r"]) > np.float32(b["r"]):
            continue
        v = float(np.float32(s["r"])) + INFLATE - np.linalg.norm(np.subtract(s["local"], b["local"])) - CERT_MARGIN
        best = max(best, v)
    return best


def rand_rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    return q * np.sign(np.diag(r))


def core_dist(x, c, axes, h):
    p = np.abs(axes @ (x - c)) - h
    return float(np.linalg.norm(np.maximum(p, 0.0)))


@pytest.mark.parametrize("robot", ["panda", "fetch", "baxter"])
def test_certain_hit_radius_implies_a_leaf_hit(robot):
    """Whenever the bound's centre lies within rho + kappa_g of a rounded box's
    core, some leaf of the group reaches at least CERT_MARGIN into the box
    (FP64, random boxes, random frame orientations)."""
    m = cases.robot_model(robot)
    sph = m["spheres"]
    rng = np.random.default_rng(11)
    checked = 0
    for g in m["env_groups"]:
        kappa = cert_radius(m, g)
        if kappa <= 0.0:
            continue
        b = sph[g["bound"]]
        rigid = [l for l in g["leaves"] if sph[l]["frame"] == b["frame"]
                 and np.float32(sph[l]["r"]) <= np.float32(b["r"])]
        offs = np.array([np.subtract(sph[l]["local"], b["local"]) for l in rigid])
        radii = np.array([float(np.float32(sph[l]["r"])) for l in rigid])
        for _ in range(300):
            axes = rand_rotation(rng)
            h = rng.uniform(0.0, 0.3, 3) * (rng.random(3) < 0.8)
            rho = rng.uniform(0.0, 0.1) if rng.random() < 0.5 else 0.0
            c = rng.normal(size=3) * 0.5
            # a bound centre at core distance t < rho + kappa: a point of a face
            # moved out along the face normal (or a point inside the core)
            a = rng.integers(3)
            sgn = rng.choice([-1.0, 1.0])
            s = rng.uniform(-1.0, 1.0, 3)
            s[a] = sgn
            t = rng.uniform(0.0, rho + kappa)
            x = c + axes.T @ (h * s) + axes[a] * sgn * t
            if rng.random() < 0.1:
                x = c + axes.T @ (h * rng.uniform(-1.0, 1.0, 3))
            if core_dist(x, c, axes, h) >= rho + kappa:
                continue
            q = rand_rotation(rng)
            pen = [r + INFLATE + rho - core_dist(x + q @ o, c, axes, h) for o, r in zip(offs, radii)]
            assert max(pen) > CERT_MARGIN * 0.999, (g.get("link"), max(pen))
            checked += 1
    assert checked > 1000


def _extractor():
    import sys
    robots = os.path.join(os.path.dirname(HEADERS), "robots")
    if robots not in sys.path:
        sys.path.insert(0, robots)
    import extract_robot
    return extract_robot


def test_regroup_encloses_leaves_and_rejects_bad_partitions():
    """The generator's regrouping (robots/extract_robot.py `regroup`) on the
    reference's Panda groups: new bounds enclose their leaves by at least the
    margin, groups equal to a reference group keep its bound, and partitions
    that drop a leaf or span two frames are refused."""
    X = _extractor()
    m = cases.robot_model("panda")
    base = dict(m)
    base["spheres"] = [{k: s[k] for k in ("frame", "local", "r", "link")} for s in m["spheres"] if s["src"] >= 0]
    base["env_groups"] = m["ref_env_groups"]
    base.pop("ref_env_groups")
    out = X.regroup(base, X.PANDA_CHECK_GROUPS)
    sph = out["spheres"]
    assert len(sph) == len(m["spheres"])
    for s_out, s_model in zip(sph[70:], m["spheres"][70:]):  # the committed bounds are reproducible
        assert np.allclose(s_out["local"], s_model["local"], atol=1e-9) and s_out["r"] == s_model["r"]
    for g, want in zip(out["env_groups"], m["env_groups"]):
        assert g["leaves"] == want["leaves"]
        b = sph[g["bound"]]
        for l in g["leaves"]:
            reach = np.linalg.norm(np.subtract(sph[l]["local"], b["local"])) + sph[l]["r"]
            assert reach <= b["r"] - 0.9 * X.CHECK_BOUND_MARGIN or g["bound"] < 70, (g["link"], l)
        if g["bound"] < 70:  # a reference group kept whole keeps the reference's bound
            assert any(r["bound"] == g["bound"] and r["leaves"] == g["leaves"] for r in m["ref_env_groups"])
    with pytest.raises(SystemExit):
        X.regroup(base, X.PANDA_CHECK_GROUPS[:-1])               # a leaf missing
    with pytest.raises(SystemExit):
        X.regroup(base, [X.PANDA_CHECK_GROUPS[0] + X.PANDA_CHECK_GROUPS[1]] + X.PANDA_CHECK_GROUPS[2:])  # two frames
