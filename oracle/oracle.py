"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker of the CUDA path and as the timed
CPU baseline.  See oracle.cpp for what is restated from the reference.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
ROBOTS = {"panda": 0, "fetch": 1, "baxter": 2}
ADJUDICATION_TOL_M = 1e-5

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle not built: run `make -C oracle` (or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        f32p = ctypes.POINTER(ctypes.c_float)
        f64p = ctypes.POINTER(ctypes.c_double)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        i64p = ctypes.POINTER(ctypes.c_int64)
        i32p = ctypes.POINTER(ctypes.c_int32)
        vp = ctypes.c_void_p
        L.orc_edge_n.argtypes = [f32p, f32p, ctypes.c_int, ctypes.c_int]
        L.orc_edge_samples.argtypes = [f32p, f32p, ctypes.c_int, ctypes.c_int, f32p]
        L.orc_fk.argtypes = [ctypes.c_int, f32p, f64p]
        L.orc_config_collides.argtypes = [vp, ctypes.c_int, ctypes.c_int, f32p, ctypes.c_int]
        L.orc_config_pen.argtypes = [vp, ctypes.c_int, ctypes.c_int, f32p]
        L.orc_config_pen.restype = ctypes.c_double
        L.orc_check.argtypes = [vp, ctypes.c_int, f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, u8p]
        L.orc_pair_pen.argtypes = [vp, ctypes.c_int, f32p, ctypes.c_int, i64p, ctypes.c_int,
                                   ctypes.c_int, f64p, i32p]
        L.orc_robot_num_spheres.argtypes = [ctypes.c_int]
        L.orc_pair_flops.argtypes = [vp, ctypes.c_int, f32p, ctypes.c_int, i64p, ctypes.c_int,
                                     ctypes.c_int, f64p, u8p]
        L.orc_pair_samples.argtypes = [vp, ctypes.c_int, f32p, ctypes.c_int, i64p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, u8p]
        _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def edge_n(start, end, resolution=32):
    s, e = _f32(start), _f32(end)
    return lib().orc_edge_n(_ptr(s, ctypes.c_float), _ptr(e, ctypes.c_float), len(s), resolution)


def edge_samples(start, end, resolution=32):
    """Reference sample set of one edge, [32 n, dof], index k = lane * n + round."""
    s, e = _f32(start), _f32(end)
    n = edge_n(s, e, resolution)
    out = np.zeros((32 * n, len(s)), np.float32)
    lib().orc_edge_samples(_ptr(s, ctypes.c_float), _ptr(e, ctypes.c_float), len(s), resolution,
                           _ptr(out, ctypes.c_float))
    return out


def fk(q, robot="panda"):
    q = _f32(q)
    ns = lib().orc_robot_num_spheres(ROBOTS[robot])
    out = np.zeros((ns, 3), np.float64)
    lib().orc_fk(ROBOTS[robot], _ptr(q, ctypes.c_float), _ptr(out, ctypes.c_double))
    return out


def check(envset, edges, resolution=32, precision=64, nthreads=None, robot="panda"):
    """Verdicts uint8 [E, N] (1 = collision) with the reference's literal semantics."""
    edges = _f32(edges)
    E = edges.shape[0]
    out = np.zeros((E, envset.num_envs), np.uint8)
    soa = envset.as_ctypes()
    nt = nthreads or os.cpu_count() or 1
    rc = lib().orc_check(ctypes.byref(soa), ROBOTS[robot], _ptr(edges, ctypes.c_float), E, resolution,
                         precision, nt, _ptr(out, ctypes.c_uint8))
    if rc != 0:
        raise RuntimeError("orc_check failed (%d)" % rc)
    return out


def pair_pen(envset, edges, pairs, resolution=32, nthreads=None, robot="panda"):
    """FP64 penetration (m) of (edge, env) pairs and the sample index of the maximum."""
    edges = _f32(edges)
    pairs = np.ascontiguousarray(pairs, np.int64).reshape(-1, 2)
    K = len(pairs)
    pen = np.zeros(K, np.float64)
    arg = np.zeros(K, np.int32)
    if K == 0:
        return pen, arg
    soa = envset.as_ctypes()
    nt = nthreads or os.cpu_count() or 1
    lib().orc_pair_pen(ctypes.byref(soa), ROBOTS[robot], _ptr(edges, ctypes.c_float), resolution,
                       _ptr(pairs, ctypes.c_int64), K, nt, _ptr(pen, ctypes.c_double),
                       _ptr(arg, ctypes.c_int32))
    return pen, arg


def config_collides(envset, env, q, precision=64, robot="panda"):
    q = _f32(q)
    soa = envset.as_ctypes()
    return bool(lib().orc_config_collides(ctypes.byref(soa), env, ROBOTS[robot],
                                          _ptr(q, ctypes.c_float), precision))


def config_pen(envset, env, q, robot="panda"):
    q = _f32(q)
    soa = envset.as_ctypes()
    return lib().orc_config_pen(ctypes.byref(soa), env, ROBOTS[robot], _ptr(q, ctypes.c_float))


def adjudicate(envset, edges, got, want, resolution=32, robot="panda", tol=ADJUDICATION_TOL_M):
    """Compare verdict matrices [E, N]; returns (num_mismatch, num_adjudicated, bad_pairs).

    A mismatch is adjudicated (tolerated) when the FP64 penetration of the pair
    lies within tol metres of contact; the rest are out-of-tolerance."""
    got = np.asarray(got).astype(bool)
    want = np.asarray(want).astype(bool)
    e_idx, v_idx = np.nonzero(got != want)
    if len(e_idx) == 0:
        return 0, 0, np.zeros((0, 2), np.int64)
    pairs = np.stack([e_idx, v_idx], 1).astype(np.int64)
    pen, _ = pair_pen(envset, edges, pairs, resolution, robot=robot)
    ok = np.abs(pen) <= tol
    return len(pairs), int(ok.sum()), pairs[~ok]


def pair_flops(envset, edges, pairs, resolution=32, nthreads=None, robot="panda"):
    """Algorithmic FLOPs of (edge, env) pairs in the reference's plain order, and
    their FP32 verdicts (the unit of the roofline's achieved FLOP/s)."""
    edges = _f32(edges)
    pairs = np.ascontiguousarray(pairs, np.int64).reshape(-1, 2)
    K = len(pairs)
    fl = np.zeros(K, np.float64)
    v = np.zeros(K, np.uint8)
    soa = envset.as_ctypes()
    nt = nthreads or os.cpu_count() or 1
    lib().orc_pair_flops(ctypes.byref(soa), ROBOTS[robot], _ptr(edges, ctypes.c_float), resolution,
                         _ptr(pairs, ctypes.c_int64), K, nt, _ptr(fl, ctypes.c_double), _ptr(v, ctypes.c_uint8))
    return fl, v


def pair_samples(envset, edges, pairs, resolution=32, max_samples=None, precision=64, nthreads=None, robot="panda"):
    """Per-sample verdicts uint8 [K, max_samples] of (edge, env) pairs: 1 collides, 0 free,
    2 past the pair's 32 n samples; sample index j = lane * n + round."""
    edges = _f32(edges)
    pairs = np.ascontiguousarray(pairs, np.int64).reshape(-1, 2)
    K = len(pairs)
    if max_samples is None:
        max_samples = 32 * max([edge_n(edges[e, 0], edges[e, 1], resolution) for e in set(pairs[:, 0].tolist())] + [1])
    out = np.full((K, max_samples), 2, np.uint8)
    if K == 0:
        return out
    soa = envset.as_ctypes()
    nt = nthreads or os.cpu_count() or 1
    lib().orc_pair_samples(ctypes.byref(soa), ROBOTS[robot], _ptr(edges, ctypes.c_float), resolution,
                           _ptr(pairs, ctypes.c_int64), K, max_samples, precision, nt, _ptr(out, ctypes.c_uint8))
    return out
