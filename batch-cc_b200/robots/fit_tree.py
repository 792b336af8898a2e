"""Kinematic-tree fitting for robots whose reference FK is generated SSA code
(Fetch, Baxter: src/utils.cuh fkcc<Fetch> :10382-24992, fkcc<Baxter>
:24994-38241).

The generated function is read as TEXT: `auto NAME = EXPR;` statements (FP64
arithmetic on the joint values) interleaved with check blocks
`if (/*link*/ sphere_environment_in_collision(environment, x, y, z, r)) {...}`
and `if (/*a vs. b*/ sphere_sphere_self_collision(8 args)) {...}`.  The
statements are evaluated with numpy to obtain every referenced sphere centre
as a function of q.  From those samples this module fits this project's own
robot model -- a kinematic tree of revolute / prismatic joints:

    frame[k + 1] = frame[parent[k]] * G_k * J_k(q_k),  J = Rz(q) or Tz(q)
    sphere centre = frame[f] * local

by (1) finding the joints each sphere depends on (the deepest one carries the
sphere, the deepest other one of its body's spheres is the joint's parent),
(2) fitting, at q = 0, the rigid motion of each joint's subtree for a step of
that joint alone (Kabsch), which gives the joint's axis, pivot and type.  The
caller verifies that the fitted tree reproduces the generated centres.
"""
import re

import numpy as np


def strip_line_comments(text):
    return "\n".join(l.split("//", 1)[0] for l in text.split("\n"))


def parse_ssa(body):
    """-> (statements [(name, expr)], env_groups, self_groups) in code order."""
    s = strip_line_comments(body)
    i, n = 0, len(s)
    depth = 0
    stmts, env, slf = [], [], []

    def args_of(cond):
        m = re.search(r"(sphere_environment_in_collision|sphere_sphere_self_collision)\s*\((.*)\)\s*$", cond, re.S)
        return m.group(1), [x.strip() for x in m.group(2).split(",")]

    while i < n:
        c = s[i]
        if c.isspace():
            i += 1
            continue
        if s.startswith("auto ", i):
            j = s.index(";", i)
            name, expr = s[i + 5:j].split("=", 1)
            stmts.append((name.strip(), " ".join(expr.split())))
            i = j + 1
            continue
        if s.startswith("if", i) and s[i + 2:].lstrip().startswith("("):
            k = s.index("(", i)
            d, j = 0, k
            while True:
                if s[j] == "(":
                    d += 1
                elif s[j] == ")":
                    d -= 1
                    if d == 0:
                        break
                j += 1
            cond = s[k + 1:j]
            label = None
            cm = re.match(r"\s*/\*(.*?)\*/", cond)
            if cm:
                label = cm.group(1).strip()
                cond = cond[cm.end():]
            kind, a = args_of(cond)
            if kind == "sphere_environment_in_collision":
                sph = tuple(a[1:5])
                if depth == 0:
                    env.append({"link": label, "bound": sph, "leaves": []})
                else:
                    env[-1]["leaves"].append(sph)
            else:
                pa, pb = tuple(a[0:4]), tuple(a[4:8])
                if depth == 0:
                    slf.append({"links": label.split(" vs. ") if label else None, "bound": [pa, pb], "pairs": []})
                else:
                    slf[-1]["pairs"].append([pa, pb])
            i = j + 1
            continue
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
        i += 1
    return stmts, env, slf


def make_evaluator(stmts, qname="q"):
    """Vectorised FP64 evaluator: q [B, dof] -> dict name -> [B] values."""
    code = ["def fk(q):"]
    for name, expr in stmts:
        e = re.sub(r"\b%s\[(\d+)\]" % qname, r"q[:, \1]", expr)
        e = re.sub(r"\bsin\(", "np.sin(", e)
        e = re.sub(r"\bcos\(", "np.cos(", e)
        code.append("    %s = %s" % (name, e))
    code.append("    return locals()")
    ns = {"np": np}
    exec("\n".join(code), ns)
    return ns["fk"]


def is_literal(tok):
    return re.match(r"^-?[\d.]", tok) is not None


def centres(fk, keys, q):
    """Sphere centres [len(keys), B, 3] of the generated code at q [B, dof]."""
    vals = fk(q.astype(np.float64))
    out = np.zeros((len(keys), q.shape[0], 3))
    for s, k in enumerate(keys):
        for a in range(3):
            t = k[a]
            out[s, :, a] = float(t) if is_literal(t) else vals[t]
    return out


def kabsch(P, Q):
    """Rigid (R, t) minimising |R P + t - Q| (P, Q: [m, 3])."""
    pc, qc = P.mean(0), Q.mean(0)
    H = (P - pc).T @ (Q - qc)
    U, _, Vt = np.linalg.svd(H)
    D = np.diag([1, 1, np.sign(np.linalg.det(Vt.T @ U.T))])
    R = Vt.T @ D @ U.T
    return R, qc - R @ pc


def hom(R, t):
    T = np.eye(4)
    T[:3, :3] = R
    T[:3, 3] = t
    return T


def fit_tree(fk, keys, dof, rng):
    """Fit the tree; returns (joints, body of each sphere, centres at q = 0)."""
    S = len(keys)
    base = centres(fk, keys, np.zeros((1, dof)))[:, 0, :]
    # (1) dependencies by finite differences at a few random configurations
    deps = [set() for _ in range(S)]
    for _ in range(3):
        q = rng.uniform(-2.0, 2.0, (1, dof))
        c0 = centres(fk, keys, q)[:, 0, :]
        for j in range(dof):
            dq = q.copy()
            dq[0, j] += 1e-3
            d = np.abs(centres(fk, keys, dq)[:, 0, :] - c0).max(1)
            for s in np.nonzero(d > 1e-9)[0]:
                deps[s].add(j)
    body = [max(d) if d else -1 for d in deps]
    parent = []
    for j in range(dof):
        ds = [deps[s] - {j} for s in range(S) if body[s] == j]
        if not ds:
            raise SystemExit("joint %d carries no sphere; cannot observe it" % j)
        anc = set().union(*ds)
        parent.append(max(anc) if anc else -1)
    sub = {j: [s for s in range(S) if j in deps[s]] for j in range(dof)}

    joints = []
    for j in range(dof):
        p = parent[j]
        # Every sphere of joint j's subtree moves rigidly with +th of q_j; at
        # q = 0 all bodies are in their reference pose, so the fitted motion
        # is the joint's screw in world (= reference) coordinates.
        ids = sub[j]
        P = base[ids]
        if len(ids) < 3 or np.linalg.matrix_rank(P - P.mean(0), tol=1e-6) < 2:
            raise SystemExit("joint %d moves too few non-collinear spheres (%d)" % (j, len(ids)))
        th = 0.7
        qb = np.zeros(dof)
        qb[j] = th
        Q = centres(fk, [keys[i] for i in ids], qb[None])[:, 0, :]
        R, t = kabsch(P, Q)
        ang = np.arccos(np.clip((np.trace(R) - 1) / 2, -1, 1))
        if ang < 1e-6:  # prismatic: pure translation along the axis
            axis = t / th
            if abs(np.linalg.norm(axis) - 1) > 1e-6:
                raise SystemExit("joint %d: translation %g per unit" % (j, np.linalg.norm(axis)))
            joints.append({"type": "prismatic", "axis": axis, "pivot": np.zeros(3), "parent": p})
            continue
        w = np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0], R[1, 0] - R[0, 1]]) / (2 * np.sin(ang))
        if abs(ang - th) > 1e-6:
            raise SystemExit("joint %d: rotation %g for %g" % (j, ang, th))
        # pivot: (I - R) c = t, least squares (the axis direction is free)
        c = np.linalg.lstsq(np.eye(3) - R, t, rcond=None)[0]
        joints.append({"type": "revolute", "axis": w / np.linalg.norm(w), "pivot": c, "parent": p})
    return joints, body, base


def z_to(axis):
    """Rotation taking +z to the unit vector `axis`."""
    z = np.array([0.0, 0.0, 1.0])
    v = np.cross(z, axis)
    c = float(z @ axis)
    if np.linalg.norm(v) < 1e-12:
        return np.eye(3) if c > 0 else np.diag([1.0, -1.0, -1.0])
    vx = np.array([[0, -v[2], v[1]], [v[2], 0, -v[0]], [-v[1], v[0], 0]])
    return np.eye(3) + vx + vx @ vx * (1.0 / (1.0 + c))


def to_model(joints, body, base):
    """Express the fitted tree in the F_k * J(q) form of the robot tables.

    With F_k = T(pivot_k) Rot(z -> axis_k) (world pose of joint k's axis frame at
    q = 0), frame'[k+1] = frame'[parent+1] * (F_parent^-1 F_k) * J(q_k) and a
    sphere on body k has local offset F_k^-1 * centre(q = 0)."""
    F = [hom(z_to(jt["axis"]), jt["pivot"]) for jt in joints]
    out = []
    for k, jt in enumerate(joints):
        Fp = np.eye(4) if jt["parent"] < 0 else F[jt["parent"]]
        G = np.linalg.inv(Fp) @ F[k]
        out.append({"tf": G[:3, :].ravel().tolist(), "type": jt["type"], "parent_frame": jt["parent"] + 1})
    local = []
    for s in range(len(body)):
        b = body[s]
        Fi = np.eye(4) if b < 0 else np.linalg.inv(F[b])
        local.append((Fi @ np.append(base[s], 1.0))[:3])
    frames = [b + 1 for b in body]
    return out, frames, local


def chain_centres(model_joints, frames, local, q):
    """FP64 evaluation of the table model at one q (for verification)."""
    T = batch_frames(model_joints, np.asarray(q, float)[None])
    return np.array([(T[f, 0] @ np.append(l, 1.0))[:3] for f, l in zip(frames, local)])


def batch_frames(model_joints, q):
    """FP64 frames [dof + 1, B, 4, 4] of the table model for a batch q [B, dof]."""
    B, dof = q.shape
    T = np.zeros((dof + 1, B, 4, 4))
    T[0] = np.eye(4)
    for k, jt in enumerate(model_joints):
        G = np.eye(4)
        G[:3, :] = np.array(jt["tf"]).reshape(3, 4)
        J = np.tile(np.eye(4), (B, 1, 1))
        if jt["type"] == "revolute":
            c, s = np.cos(q[:, k]), np.sin(q[:, k])
            J[:, 0, 0], J[:, 0, 1], J[:, 1, 0], J[:, 1, 1] = c, -s, s, c
        else:
            J[:, 2, 3] = q[:, k]
        T[k + 1] = T[jt["parent_frame"]] @ G @ J
    return T


def path_joints(model_joints, fa, fb):
    """Joints whose value changes the relative pose of frames fa and fb."""
    def chain(f):
        out = []
        while f > 0:
            out.append(f - 1)
            f = model_joints[f - 1]["parent_frame"]
        return out
    return sorted(set(chain(fa)) ^ set(chain(fb)))


def max_distance(model_joints, fa, la, fb, lb, dof, grid=721):
    """Max over q of |centre(fa, la) - centre(fb, lb)| (frames in the tree).

    Only the joints on the path between the two frames matter; they are swept
    over a full turn on a grid and the best grid points are refined by a local
    search, so the value is the supremum to well below a micrometre."""
    from scipy.optimize import minimize

    js = path_joints(model_joints, fa, fb)
    for j in js:
        if model_joints[j]["type"] != "revolute":
            raise SystemExit("prismatic joint %d between a bound and its leaf" % j)
    if not js:
        T = batch_frames(model_joints, np.zeros((1, dof)))
        return float(np.linalg.norm(T[fa, 0] @ np.append(la, 1.0) - T[fb, 0] @ np.append(lb, 1.0)))
    if len(js) > 2:
        raise SystemExit("bound and leaf %d joints apart" % len(js))

    def dist(vals):
        vals = np.atleast_2d(vals)
        q = np.zeros((len(vals), dof))
        q[:, js] = vals
        T = batch_frames(model_joints, q)
        return np.linalg.norm(T[fa] @ np.append(la, 1.0) - T[fb] @ np.append(lb, 1.0), axis=1)

    axes = np.linspace(-np.pi, np.pi, grid)
    if len(js) == 1:
        pts = axes[:, None]
    else:
        pts = np.stack(np.meshgrid(axes, axes, indexing="ij"), -1).reshape(-1, 2)
    d = np.concatenate([dist(pts[i:i + 65536]) for i in range(0, len(pts), 65536)])
    best = float(d.max())
    for i in np.argsort(d)[-8:]:
        r = minimize(lambda v: -dist(v)[0], pts[i], method="Nelder-Mead",
                     options={"xatol": 1e-10, "fatol": 1e-14, "maxiter": 4000})
        best = max(best, -float(r.fun))
    return best


def enclosing_sphere(centres_, radii):
    """A sphere containing every (centre, radius) ball: the current sphere is
    grown to the span of itself and each ball outside it (exact for two balls)."""
    c = np.array(centres_[0], float)
    r = float(radii[0])
    for _ in range(2):
        for x, rx in zip(centres_, radii):
            x = np.asarray(x, float)
            d = np.linalg.norm(x - c)
            if d + rx <= r:
                continue
            if d < 1e-15:
                r = rx
                continue
            far = c - (x - c) / d * r        # the point of the current sphere farthest from x
            near = x + (x - c) / d * rx      # the point of x's ball farthest from c
            c = 0.5 * (far + near)
            r = 0.5 * np.linalg.norm(near - far)
    return c, r


def smallest_enclosing_sphere(centres_, radii):
    """The smallest sphere containing every (centre, radius) ball: the centre c
    minimises max_i |c - x_i| + r_i (a convex function), found by Nelder-Mead
    from three starts; the radius is that maximum at the centre found, so the
    sphere contains every ball whatever the optimiser's accuracy."""
    from scipy.optimize import minimize

    pts = np.asarray(centres_, float)
    r = np.asarray(radii, float)

    def reach(c):
        return float((np.linalg.norm(pts - c, axis=1) + r).max())

    best = None
    for start in (pts.mean(0), 0.5 * (pts.min(0) + pts.max(0)), pts[int(np.argmax(r))]):
        res = minimize(reach, start, method="Nelder-Mead",
                       options={"xatol": 1e-10, "fatol": 1e-12, "maxiter": 20000})
        if best is None or reach(res.x) < reach(best):
            best = res.x
    return best, reach(best)
