"""Seeded synthetic workloads for the batch edge collision checker.

The reference publishes no benchmark data; its drivers build environments from
MotionBenchMaker problem files and edges from a Halton sequence
(scripts/batch_cc_mbm.cpp:96-139).  The workloads here are seeded synthetic
stand-ins with the primitive kinds, counts and size laws of the five benchmark
configurations:

* ``plain``      panda, 100 envs x 1000 edges; per env 8 spheres, 8 cuboids,
                 4 cylinders (stored as capsules); endpoints uniform in limits.
* ``uneven``     panda, 1000 envs x 10000 edges; U{8..64} primitives per env
                 (40 % cuboid, 40 % sphere, 20 % cylinder->capsule); edges of
                 log-uniform length 0.05-2.0 rad.
* ``multi``      fetch / baxter, 500 envs x 5000 edges, U{16..256} primitives,
                 workspace x1.5.
* ``stress``     panda, 10000 envs x 100000 edges, U{8..128} primitives, with an
                 obstacle-density multiplier.
Sizes: sphere r U[0.05,0.15]; cuboid half-extents U[0.02,0.3] with random yaw;
cylinder r U[0.03,0.1], length U[0.1,0.6], Euler XYZ U[-pi,pi]^3; centres
U([-0.8,0.8]^2 x [0,1.2]) m.

Cuboid axes and capsule endpoints follow the reference shape factory
(src/collision/factory.hh): rotation Rz(phi) Ry(theta) Rx(rho); a cylinder of
length L about centre c becomes the capsule from c + R (0,0,L/2) to
c + R (0,0,-L/2) with rdv = 1 / |v|^2 (factory.hh:165-185, 118-129); drivers
store cylinders as capsules (scripts/batch_cc_mbm.cpp:46-59).
"""
import math

import numpy as np

from .envs import EnvSet

# Joint-limit scale q = u * s_m + s_a (src/Robots.hh:17-41, :72-98, :128-166).
LIMITS = {
    "panda": (np.array([5.9342, 3.6652, 5.9342, 3.2289, 5.9342, 3.9095999999999997, 5.9342], np.float32),
              np.array([-2.9671, -1.8326, -2.9671, -3.1416, -2.9671, -0.0873, -2.9671], np.float32)),
    "fetch": (np.array([0.38615, 3.2112, 2.739, 6.28318, 4.502, 6.28318, 4.32, 6.28318], np.float32),
              np.array([0.0, -1.6056, -1.221, -3.14159, -2.251, -3.14159, -2.16, -3.14159], np.float32)),
    "baxter": (np.array([3.40335987756, 3.194, 6.10835987756, 2.6679999999999997, 6.118, 3.66479632679, 6.118] * 2, np.float32),
               np.array([-1.70167993878, -2.147, -3.05417993878, -0.05, -3.059, -1.57079632679, -3.059] * 2, np.float32)),
}
DOF = {"panda": 7, "fetch": 8, "baxter": 14}

WORKLOADS = {
    "plain": dict(robot="panda", envs=100, edges=1000, prims="fixed", edge_law="uniform",
                  box=(0.8, 0.8, 0.0, 1.2), density=1.0),
    "uneven": dict(robot="panda", envs=1000, edges=10000, prims=(8, 64), edge_law="loglen",
                   box=(0.8, 0.8, 0.0, 1.2), density=1.0),
    "multi_fetch": dict(robot="fetch", envs=500, edges=5000, prims=(16, 256), edge_law="loglen",
                        box=(1.2, 1.2, 0.0, 1.8), density=1.0),
    "multi_baxter": dict(robot="baxter", envs=500, edges=5000, prims=(16, 256), edge_law="loglen",
                         box=(1.2, 1.2, 0.0, 1.8), density=1.0),
    "stress": dict(robot="panda", envs=10000, edges=100000, prims=(8, 128), edge_law="loglen",
                   box=(0.8, 0.8, 0.0, 1.2), density=0.1, shell=True),
}

# Stress workload obstacle placement: a fraction `density` of obstacle centres
# lies in the arm's reachable shell (distance 0.45-0.85 m from the shoulder,
# above the floor), the rest beyond reach (1.05-1.6 m).  `density` is the
# concentration multiplier tuned for a ~40 % colliding-edge fraction.
SHOULDER = np.array([0.0, 0.0, 0.333])
SHELL = (0.45, 0.85)
OUTER = (1.05, 1.6)


def euler_xyz_matrix(rho, theta, phi):
    """Rz(phi) @ Ry(theta) @ Rx(rho), float32 like the reference factory's Eigen floats."""
    cr, sr = np.cos(rho), np.sin(rho)
    ct, st = np.cos(theta), np.sin(theta)
    cp, sp = np.cos(phi), np.sin(phi)
    one, zero = np.ones_like(rho), np.zeros_like(rho)
    rx = np.stack([np.stack([one, zero, zero], -1), np.stack([zero, cr, -sr], -1),
                   np.stack([zero, sr, cr], -1)], -2)
    ry = np.stack([np.stack([ct, zero, st], -1), np.stack([zero, one, zero], -1),
                   np.stack([-st, zero, ct], -1)], -2)
    rz = np.stack([np.stack([cp, -sp, zero], -1), np.stack([sp, cp, zero], -1),
                   np.stack([zero, zero, one], -1)], -2)
    return (rz @ ry @ rx).astype(np.float32)


def make_cuboids(centre, euler, half):
    """Cuboid records [m, 15] from centres, Euler XYZ angles and half-extents."""
    R = euler_xyz_matrix(euler[:, 0], euler[:, 1], euler[:, 2])
    rec = np.zeros((len(centre), 15), np.float32)
    rec[:, 0:3] = centre
    rec[:, 3:6] = R[:, :, 0]
    rec[:, 6:9] = R[:, :, 1]
    rec[:, 9:12] = R[:, :, 2]
    rec[:, 12:15] = half
    return rec


def make_capsules(centre, euler, radius, length):
    """Capsule records [m, 8] of cylinders given by centre, Euler XYZ, radius, length."""
    R = euler_xyz_matrix(euler[:, 0], euler[:, 1], euler[:, 2])
    half = (length.astype(np.float32) / np.float32(2))
    ax = R[:, :, 2] * half[:, None]
    p1 = (centre.astype(np.float32) + ax).astype(np.float32)
    p2 = (centre.astype(np.float32) - ax).astype(np.float32)
    v = (p2 - p1).astype(np.float32)
    dot = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2]).astype(np.float32)
    with np.errstate(divide="ignore"):
        rdv = (1.0 / dot.astype(np.float64)).astype(np.float32)
    rec = np.zeros((len(centre), 8), np.float32)
    rec[:, 0:3] = p1
    rec[:, 3:6] = v
    rec[:, 6] = radius
    rec[:, 7] = rdv
    return rec


def make_spheres(centre, radius):
    rec = np.zeros((len(centre), 4), np.float32)
    rec[:, 0:3] = centre
    rec[:, 3] = radius
    return rec


def gen_envs(name, num_envs=None, seed=0, density=None):
    w = WORKLOADS[name]
    n = w["envs"] if num_envs is None else num_envs
    dens = w["density"] if density is None else density
    rng = np.random.default_rng(np.random.SeedSequence([seed, 1, hash_name(name)]))
    bx, by, z0, z1 = w["box"]
    envs = []
    for _ in range(n):
        if w["prims"] == "fixed":
            ns, nb, nc = 8, 8, 4
        else:
            lo, hi = w["prims"]
            p = int(rng.integers(lo, hi + 1))
            kind = rng.choice(3, size=p, p=[0.4, 0.4, 0.2])
            nb, ns, nc = int((kind == 0).sum()), int((kind == 1).sum()), int((kind == 2).sum())

        def centres(m):
            if not w.get("shell"):
                return np.stack([rng.uniform(-bx, bx, m), rng.uniform(-by, by, m), rng.uniform(z0, z1, m)], -1)
            d = rng.normal(size=(m, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            d[:, 2] = np.abs(d[:, 2]) * 0.8 - 0.2  # mostly above the shoulder plane
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            inner = rng.uniform(0, 1, m) < dens
            rad = np.where(inner, rng.uniform(*SHELL, m), rng.uniform(*OUTER, m))
            c = SHOULDER + d * rad[:, None]
            c[:, 2] = np.maximum(c[:, 2], 0.0)
            return c
        sph = make_spheres(centres(ns), rng.uniform(0.05, 0.15, ns))
        yaw = rng.uniform(-math.pi, math.pi, nb)
        eul = np.stack([np.zeros(nb), np.zeros(nb), yaw], -1)
        cub = make_cuboids(centres(nb), eul, rng.uniform(0.02, 0.3, (nb, 3)))
        eulc = rng.uniform(-math.pi, math.pi, (nc, 3))
        cap = make_capsules(centres(nc), eulc, rng.uniform(0.03, 0.1, nc), rng.uniform(0.1, 0.6, nc))
        envs.append({"spheres": sph, "cuboids": cub, "capsules": cap})
    return EnvSet.from_lists(envs)


def hash_name(name):
    return sum((i + 1) * ord(c) for i, c in enumerate(name)) % 100003


def gen_edges(name, num_edges=None, seed=0):
    """Edges float32 [E, 2, dof] (start, end) in the reference's AoS layout."""
    w = WORKLOADS[name]
    robot = w["robot"]
    E = w["edges"] if num_edges is None else num_edges
    s_m, s_a = LIMITS[robot]
    lo = s_a.astype(np.float64)
    hi = (s_a + s_m).astype(np.float64)
    dof = DOF[robot]
    rng = np.random.default_rng(np.random.SeedSequence([seed, 2, hash_name(name)]))
    if w["edge_law"] == "uniform":
        start = rng.uniform(lo, hi, (E, dof))
        end = rng.uniform(lo, hi, (E, dof))
    else:
        start = rng.uniform(lo, hi, (E, dof))
        end = np.empty_like(start)
        todo = np.arange(E)
        while len(todo):
            d = rng.normal(size=(len(todo), dof))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            L = np.exp(rng.uniform(math.log(0.05), math.log(2.0), len(todo)))
            cand = start[todo] + d * L[:, None]
            ok = np.all((cand >= lo) & (cand <= hi), axis=1)
            end[todo[ok]] = cand[ok]
            todo = todo[~ok]
    return np.ascontiguousarray(np.stack([start, end], 1).astype(np.float32))


def robot_of(name):
    return WORKLOADS[name]["robot"]
