"""ctypes binding of the reference harness (oracle/_ref/libbcc_ref.so).

TEST INFRASTRUCTURE ONLY.  The library is the reference's own src/batch_cc.cu,
unmodified, compiled for sm_100a by `make -C oracle ref` in the development
container (see ref_harness.cu); it travels to the GPU box as a built file.
Used by the GPU parity tests (verdicts of the reference CUDA path, the
reference kernel's exact sample set) and by bench.py's reference arm.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libbcc_ref.so")
PROBE_ROUNDS = 16

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("reference harness not built (make -C oracle ref, needs the reference tree)")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        f32p = ctypes.POINTER(ctypes.c_float)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.ref_check.argtypes = [ctypes.c_int, vp, f32p, ctypes.c_int, ctypes.c_int, u8p, ctypes.c_int]
        L.ref_time.argtypes = [ctypes.c_int, vp, f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, f32p, u8p]
        L.ref_probe_samples.argtypes = [f32p, ctypes.c_int, ctypes.c_int, f32p, i32p]
        _lib = L
    return _lib


ROBOTS = {"panda": 0, "fetch": 1, "baxter": 2}


def check(envset, edges, resolution=32, quiet=True, robot="panda"):
    """Verdicts [E, N] from batch_cc::batch_cc<Robot> (the reference public API)."""
    edges = np.ascontiguousarray(edges, np.float32)
    E = edges.shape[0]
    out = np.zeros((E, envset.num_envs), np.uint8)
    soa = envset.as_ctypes()
    rc = lib().ref_check(ROBOTS[robot], ctypes.byref(soa), edges.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), E,
                         resolution, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), int(quiet))
    if rc != 0:
        raise RuntimeError("reference batch_cc failed with CUDA error %d" % rc)
    return out


def time_kernel(envset, edges, resolution=32, iters=3, robot="panda"):
    """(mean kernel ms, verdicts [E, N]) of the reference kernel, CUDA-event timed."""
    edges = np.ascontiguousarray(edges, np.float32)
    E = edges.shape[0]
    out = np.zeros((E, envset.num_envs), np.uint8)
    ms = ctypes.c_float(0)
    soa = envset.as_ctypes()
    rc = lib().ref_time(ROBOTS[robot], ctypes.byref(soa), edges.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                        E, resolution, iters, ctypes.byref(ms), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    if rc != 0:
        raise RuntimeError("reference kernel failed with CUDA error %d" % rc)
    return float(ms.value), out


def probe_samples(edges, resolution=32):
    """Configurations the reference kernel checks: ([E, 32, 16, 7] lane x round, counts [E, 32])."""
    edges = np.ascontiguousarray(edges, np.float32)
    E = edges.shape[0]
    out = np.zeros((E, 32, PROBE_ROUNDS, 7), np.float32)
    cnt = np.zeros((E, 32), np.int32)
    rc = lib().ref_probe_samples(edges.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), E, resolution,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                 cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    if rc != 0:
        raise RuntimeError("reference probe failed with CUDA error %d" % rc)
    return out, cnt
