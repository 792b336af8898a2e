"""CPU tests of the host side of the C ABI: exported symbols, validation, and
the rounded-box packing that lets one device predicate serve every primitive
kind (compared with exact FP64 distances to the original primitives)."""
import ctypes
import os
import re

import numpy as np
import pytest

from bcc import EnvSet, workload
from bcc import lib as bcclib
from bcc.workload import make_capsules, make_cuboids, make_spheres

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "bcc.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bcc_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = bcclib.lib()
    names = declared_functions()
    assert "bcc_check" in names and "bcc_upload_envs" in names
    for n in names:
        assert hasattr(L, n), n


def pack(envset):
    L = bcclib.lib()
    soa = envset.as_ctypes()
    n = ctypes.c_int64(0)
    mp = ctypes.c_int32(0)
    st = L.bcc_pack_envs(ctypes.byref(soa), None, None, ctypes.byref(n), ctypes.byref(mp))
    if st != 0:
        return st, None, None
    rec = np.zeros((n.value, 20), np.float32)
    off = np.zeros(envset.num_envs + 1, np.int32)
    st = L.bcc_pack_envs(ctypes.byref(soa), rec.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                         off.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(n), ctypes.byref(mp))
    return st, rec, off


def rounded_box_dist(rec, p):
    d = p - rec[:3].astype(np.float64)
    s = 0.0
    for i in range(3):
        a = rec[4 + 4 * i:7 + 4 * i].astype(np.float64)
        h = float(rec[7 + 4 * i])
        s += max(abs(a @ d) - h, 0.0) ** 2
    return np.sqrt(s) - float(rec[3])


def seg_dist(p, a, v):
    t = np.clip((p - a) @ v / (v @ v), 0, 1) if v @ v > 0 else 0.0
    return np.linalg.norm(p - (a + t * v))


def box_dist(p, c, A, h):
    loc = A @ (p - c)
    return np.linalg.norm(np.maximum(np.abs(loc) - h, 0))


def test_rounded_box_packing_matches_exact_distances():
    rng = np.random.default_rng(0)
    sph = make_spheres(rng.uniform(-1, 1, (5, 3)), rng.uniform(0.05, 0.15, 5))
    cap = make_capsules(rng.uniform(-1, 1, (5, 3)), rng.uniform(-np.pi, np.pi, (5, 3)),
                        rng.uniform(0.03, 0.1, 5), rng.uniform(0.0, 0.6, 5))
    cub = make_cuboids(rng.uniform(-1, 1, (5, 3)), rng.uniform(-np.pi, np.pi, (5, 3)), rng.uniform(0.02, 0.3, (5, 3)))
    zc = cap.copy()
    zc[:, 3:5] = 0.0
    zc[:, 7] = 1.0 / (zc[:, 5].astype(np.float64) ** 2)
    zb = make_cuboids(rng.uniform(-1, 1, (5, 3)), np.stack([np.zeros(5), np.zeros(5), rng.uniform(-3, 3, 5)], 1),
                      rng.uniform(0.02, 0.3, (5, 3)))
    envs = EnvSet.from_lists([{"spheres": sph, "capsules": cap, "z_capsules": zc, "cuboids": cub, "z_cuboids": zb}])
    st, rec, off = pack(envs)
    assert st == 0 and list(off) == [0, 25]
    pts = rng.uniform(-1.5, 1.5, (200, 3))
    for p in pts:
        exact = [np.linalg.norm(p - s[:3]) - s[3] for s in sph]
        exact += [seg_dist(p, c[:3].astype(np.float64), c[3:6].astype(np.float64)) - c[6] for c in cap]
        exact += [seg_dist(p, c[:3].astype(np.float64), np.array([0, 0, c[5]], np.float64)) - c[6] for c in zc]
        exact += [box_dist(p, b[:3], b[3:12].reshape(3, 3).astype(np.float64), b[12:15]) for b in cub]
        exact += [box_dist(p, b[:3], b[3:12].reshape(3, 3).astype(np.float64), b[12:15]) for b in zb]
        got = [rounded_box_dist(r, p) for r in rec]
        assert np.allclose(got, exact, atol=2e-6), (np.array(got) - np.array(exact))
    # cull AABB half-size bounds every point of the primitive
    for r in rec:
        assert np.all(r[16:19] >= r[3] - 1e-7)


def test_pack_rejects_positive_count_with_null_records():
    envs = workload.gen_envs("plain", 2, seed=0)
    soa = envs.as_ctypes()
    soa.cuboids = None
    st = bcclib.lib().bcc_pack_envs(ctypes.byref(soa), None, None, None, None)
    assert st == 1  # BCC_ERR_INVALID_ARGUMENT, like ensure_ptr_count_consistent


def test_pack_limit_on_primitives_per_env():
    sph = make_spheres(np.zeros((4096, 3)), np.full(4096, 0.1))
    st, _, _ = pack(EnvSet.from_lists([{"spheres": sph}]))
    assert st == 6  # BCC_ERR_LIMIT
    st, _, off = pack(EnvSet.from_lists([{"spheres": sph[:4095]}]))
    assert st == 0 and off[-1] == 4095


def test_pack_empty_and_ragged_sets():
    envs = EnvSet.from_lists([{}, {"spheres": make_spheres(np.zeros((3, 3)), np.full(3, 0.1))}, {}])
    st, rec, off = pack(envs)
    assert st == 0 and list(off) == [0, 0, 3, 3]


def test_checker_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(bcclib.BccError):
        bcclib.Checker(0)


def test_robot_ids_of_the_binding():
    from bcc.lib import ROBOTS, _rid
    assert [_rid(r) for r in ("panda", "fetch", "baxter")] == [0, 1, 2]
    assert _rid(7) == 7  # ids pass through (an unknown one is the library's to reject)
    assert ROBOTS == {"panda": 0, "fetch": 1, "baxter": 2}


def test_opts_binding_matches_the_header():
    """The ctypes mirror of bcc_opts has the header's fields, in order, all int32."""
    text = open(os.path.join(ROOT, "include", "bcc.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    body = re.search(r"typedef struct bcc_opts \{(.*?)\} bcc_opts;", text, flags=re.S).group(1)
    fields = re.findall(r"int32_t\s+(\w+);", body)
    assert [f for f, _ in bcclib.BccOpts._fields_] == fields
    assert all(t is ctypes.c_int32 for _, t in bcclib.BccOpts._fields_)
    o = bcclib.make_opts("learned", use_graph=True, tile=0, row_cap=77)
    assert (o.order, o.use_graph, o.tile_override, o.learned_row_cap) == (bcclib.ORDERS["learned"], 1, 0, 77)
