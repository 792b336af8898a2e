"""The allocation-free entry point bcc_check_noalloc, through the C ABI.

This entry point is for callers that cannot allocate device memory (a
real-time planning thread, or a framework that owns all device memory in its
own pool); it keeps its working buffers in fixed arrays inside the library.
Here it must give the same verdicts as the regular entry point bcc_check,
within the tolerance every parity test uses (mismatches only within 1e-5 m of
contact), on two calls in a row with different edges -- the second call runs
on arrays the first one left behind.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from bcc import workload
from bcc import lib as bcclib
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    L = bcclib.lib()
    f = L.bcc_check_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [ctypes.c_int, vp, vp, ctypes.c_int32, ctypes.c_int32, vp, ctypes.c_int32, ctypes.c_int32,
                  vp, vp]
    f.restype = ctypes.c_int
    return f


def _pack(envs):
    L = bcclib.lib()
    soa = envs.as_ctypes()
    n = ctypes.c_int64(0)
    mp = ctypes.c_int32(0)
    assert L.bcc_pack_envs(ctypes.byref(soa), None, None, ctypes.byref(n), ctypes.byref(mp)) == 0
    rec = np.zeros((max(n.value, 1), 20), np.float32)
    off = np.zeros(envs.num_envs + 1, np.int32)
    assert L.bcc_pack_envs(ctypes.byref(soa), rec.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                           off.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(n),
                           ctypes.byref(mp)) == 0
    return rec, off, mp.value


@pytest.mark.parametrize("name,nenv,nedge", [("uneven", 24, 96), ("multi_fetch", 12, 40), ("multi_baxter", 10, 40)])
def test_noalloc_matches_bcc_check_twice(name, nenv, nedge):
    import torch

    robot = workload.robot_of(name)
    rid = bcclib.ROBOTS[robot]
    envs = workload.gen_envs(name, nenv, seed=41)
    rec, off, max_prims = _pack(envs)
    d_rec = torch.from_numpy(rec).cuda()
    d_off = torch.from_numpy(off).cuda()
    fn = _noalloc_fn()
    chk = bcclib.Checker(0)
    chk.upload(envs)
    for call, seed in enumerate((42, 43)):
        edges = workload.gen_edges(name, nedge, seed=seed)
        want = chk.check(edges, robot=robot)
        d_edges = torch.from_numpy(edges).cuda()
        d_res = torch.full((len(edges), envs.num_envs), 7, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        st = fn(rid, d_rec.data_ptr(), d_off.data_ptr(), envs.num_envs, max_prims, d_edges.data_ptr(), len(edges),
                32, d_res.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == 0, "call %d returned status %d" % (call, st)
        torch.cuda.synchronize()
        got = d_res.cpu().numpy()
        assert set(np.unique(got)) <= {0, 1}
        n_mis, n_adj, bad = orc.adjudicate(envs, edges, got, want, robot=robot)
        assert len(bad) == 0, "call %d: %d mismatches beyond 1e-5 m of contact" % (call, len(bad))
    chk.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch

    envs = workload.gen_envs("uneven", 2, seed=44)
    rec, off, max_prims = _pack(envs)
    d_rec = torch.from_numpy(rec).cuda()
    d_off = torch.from_numpy(off).cuda()
    fn = _noalloc_fn()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # 1025 edges: more than the fixed working arrays hold.
    edges = workload.gen_edges("uneven", 1025, seed=44)
    d_edges = torch.from_numpy(edges).cuda()
    d_res = torch.zeros((1025, 2), dtype=torch.uint8, device="cuda")
    assert fn(0, d_rec.data_ptr(), d_off.data_ptr(), 2, max_prims, d_edges.data_ptr(), 1025, 32,
              d_res.data_ptr(), stream) == 6  # BCC_ERR_LIMIT
    # 200 long edges need more than 4096 samples.
    s_m, s_a = workload.LIMITS["panda"]
    rng = np.random.default_rng(0)
    q = (rng.uniform(0, 1, (400, 7)) * s_m + s_a).astype(np.float32)
    long_edges = np.ascontiguousarray(np.stack([q[:200], q[200:]], 1))
    assert sum(orc.edge_n(e[0], e[1]) * 32 for e in long_edges) > 4096
    d_edges = torch.from_numpy(long_edges).cuda()
    assert fn(0, d_rec.data_ptr(), d_off.data_ptr(), 2, max_prims, d_edges.data_ptr(), 200, 32,
              d_res.data_ptr(), stream) == 6
    # Records 4 bytes off a 16-byte boundary: refused on the host before any launch.
    d_edges = torch.from_numpy(workload.gen_edges("uneven", 8, seed=45)).cuda()
    assert fn(0, d_rec.data_ptr() + 4, d_off.data_ptr(), 2, max_prims, d_edges.data_ptr(), 8, 32,
              d_res.data_ptr(), stream) == 1  # BCC_ERR_INVALID_ARGUMENT
    torch.cuda.synchronize()
