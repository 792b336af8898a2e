"""GPU parity: the CUDA checker through the C ABI against the CPU oracle and
against the reference's own CUDA path (oracle/_ref), on seeded inputs.

Bar: every verdict mismatch must be adjudicated -- the FP64 penetration of
the pair within 1e-5 m of contact (ADJUDICATION_TOL_M); out-of-tolerance
mismatches must be 0.  The sample set is bit-exact (integer/float index work).
"""
import numpy as np
import pytest

from bcc import EnvSet, workload
from bcc.workload import make_capsules, make_cuboids, make_spheres
from oracle import oracle as orc
from oracle import ref

import cases
from bcc import lib as bcclib

pytestmark = pytest.mark.gpu

TOL = orc.ADJUDICATION_TOL_M  # 1e-5 m


def assert_parity(envs, edges, got, want, label, robot="panda"):
    n_mis, n_adj, bad = orc.adjudicate(envs, edges, got, want, tol=TOL, robot=robot)
    assert len(bad) == 0, "%s: %d mismatches, %d out of tolerance, e.g. (edge, env) %s" % (
        label, n_mis, len(bad), bad[:5].tolist())
    return n_mis


@pytest.mark.parametrize("name,nenv,nedge,seed", [
    ("plain", 16, 200, 1), ("uneven", 40, 300, 2), ("uneven", 7, 513, 3), ("stress", 25, 150, 4),
    ("multi_fetch", 16, 150, 5), ("multi_baxter", 12, 120, 6)])
def test_checker_matches_oracle(checker, name, nenv, nedge, seed):
    robot = workload.robot_of(name)
    envs = workload.gen_envs(name, nenv, seed=seed)
    edges = workload.gen_edges(name, nedge, seed=seed)
    checker.upload(envs)
    got = checker.check(edges, robot=robot)
    want = orc.check(envs, edges, precision=64, robot=robot)
    assert got.shape == want.shape
    assert_parity(envs, edges, got, want, name, robot)


def test_edge_cases(checker):
    rng = np.random.default_rng(7)
    lists = [
        {},  # empty environment
        {"spheres": make_spheres(rng.uniform(-0.6, 0.6, (1, 3)), [0.1])},
        {"capsules": make_capsules(rng.uniform(-0.6, 0.6, (3, 3)), rng.uniform(-3, 3, (3, 3)),
                                   np.full(3, 0.05), np.zeros(3))},  # zero-length capsules
        {"cuboids": make_cuboids(rng.uniform(-0.6, 0.6, (4, 3)), rng.uniform(-3, 3, (4, 3)),
                                 rng.uniform(0.02, 0.3, (4, 3)))},  # fully rotated cuboids
    ]
    zc = make_capsules(rng.uniform(-0.6, 0.6, (3, 3)), np.zeros((3, 3)), np.full(3, 0.06), np.full(3, 0.4))
    zb = make_cuboids(rng.uniform(-0.6, 0.6, (3, 3)), np.stack([np.zeros(3), np.zeros(3), [0.3, 1.0, -2.0]], 1),
                      rng.uniform(0.02, 0.2, (3, 3)))
    lists.append({"z_capsules": zc, "z_cuboids": zb, "cylinders": zc})
    envs = EnvSet.from_lists(lists)
    s_m, s_a = workload.LIMITS["panda"]
    q = (rng.uniform(0, 1, (40, 7)) * s_m + s_a).astype(np.float32)
    edges = [np.stack([q[i], q[i]]) for i in range(10)]                     # zero-length (n = 1)
    edges += [np.stack([q[i], q[i + 1]]) for i in range(10, 30)]            # long, n up to ~13
    edges += [np.stack([q[i], q[i] + 31.0 / 32.0 / np.sqrt(7)]) for i in range(30, 40)]  # step boundary
    edges = np.ascontiguousarray(np.stack(edges), np.float32)
    checker.upload(envs)
    got = checker.check(edges)
    want = orc.check(envs, edges)
    assert_parity(envs, edges, got, want, "edge cases")


def test_known_answer_contact(checker):
    """Sphere obstacle 1e-4 m beyond / inside contact with the fingertip."""
    q = np.array([0.3, -0.4, 0.2, -2.0, 0.1, 1.8, 0.5], np.float32)
    c = orc.fk(q)
    d = (c[6] - c[26]) / np.linalg.norm(c[6] - c[26])
    r_inf = 0.012000000104308128 + 0.005
    lists = [{"spheres": make_spheres((c[2] + d * (r_inf + 0.05 + g))[None], [0.05])} for g in (1e-4, -1e-4)]
    envs = EnvSet.from_lists(lists)
    checker.upload(envs)
    got = checker.check(np.stack([q, q])[None])
    assert got.tolist() == [[0, 1]]


@pytest.mark.parametrize("robot", ["fetch", "baxter"])
def test_overhanging_leaf_needs_the_bound_to_hit_somewhere(checker, robot):
    """Leaves sticking out of their bound: a leaf hit counts only when the
    bound hits SOME primitive at that sample (reference gate semantics), also
    when that primitive is not the one the leaf hits -- through the grid
    kernel, the persistent kernel and the records kernel."""
    import ctypes

    import torch

    from test_zz_no_alloc import _noalloc_fn, _pack

    q, envs, want = cases.overhang_case(robot)
    edge = np.ascontiguousarray(np.stack([q, q])[None])
    checker.upload(envs)
    old = checker.launch_config()
    try:
        for warps, persistent in ((4, 0), (8, 1)):
            checker.set_launch_config(warps=warps, persistent=persistent)
            assert checker.check(edge, robot=robot)[0].tolist() == want.tolist(), (warps, persistent)
    finally:
        checker.set_launch_config(**old)
    # the allocation-free entry point (records kernel)
    rec, off, max_prims = _pack(envs)
    d_rec, d_off = torch.from_numpy(rec).cuda(), torch.from_numpy(off).cuda()
    d_edges = torch.from_numpy(edge).cuda()
    d_res = torch.full((1, 3), 7, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    st = _noalloc_fn()(bcclib.ROBOTS[robot], d_rec.data_ptr(), d_off.data_ptr(), 3, max_prims, d_edges.data_ptr(),
                       1, 32, d_res.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    torch.cuda.synchronize()
    assert d_res.cpu().numpy()[0].tolist() == want.tolist()


def test_results_layout_and_env_permutation(checker):
    envs = workload.gen_envs("uneven", 30, seed=12)
    edges = workload.gen_edges("uneven", 100, seed=12)
    checker.upload(envs)
    a = checker.check(edges)
    perm = np.random.default_rng(0).permutation(30)
    checker.upload(envs.subset(perm))
    b = checker.check(edges)
    assert np.array_equal(a[:, perm], b)
    c = checker.check(edges[::-1].copy())
    assert np.array_equal(b[::-1], c)


def test_device_api_matches_host_api(checker):
    import torch
    envs = workload.gen_envs("uneven", 20, seed=13)
    edges = workload.gen_edges("uneven", 200, seed=13)
    checker.upload(envs)
    host = checker.check(edges)
    d_edges = torch.from_numpy(edges).cuda()
    d_res = torch.zeros((200, 20), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    checker.check_device(d_edges.data_ptr(), 200, d_res.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(d_res.cpu().numpy(), host)


def test_errors_are_reported(checker):
    from bcc.lib import BccError
    envs = workload.gen_envs("plain", 2, seed=0)
    soa_env = envs
    checker.upload(soa_env)
    with pytest.raises(BccError):
        checker.check(workload.gen_edges("plain", 4, seed=0), resolution=0)
    with pytest.raises(BccError):
        checker.check(workload.gen_edges("plain", 4, seed=0), robot=7)  # no such robot


@pytest.mark.skipif(not ref.available(), reason="reference harness not built")
def test_reference_kernel_sample_set_is_the_oracles():
    """The reference kernel's own checked configurations (probe robot) equal the
    oracle's restated discretisation bit for bit."""
    rng = np.random.default_rng(21)
    s_m, s_a = workload.LIMITS["panda"]
    q = (rng.uniform(0, 1, (120, 7)) * s_m + s_a).astype(np.float32)
    edges = [np.stack([q[i], q[i + 60]]) for i in range(60)]
    edges += list(workload.gen_edges("uneven", 60, seed=21))
    edges = np.ascontiguousarray(np.stack(edges), np.float32)
    out, cnt = ref.probe_samples(edges)
    for e in range(len(edges)):
        n = orc.edge_n(edges[e, 0], edges[e, 1])
        assert np.all(cnt[e] == n)
        S = orc.edge_samples(edges[e, 0], edges[e, 1]).reshape(32, n, 7)
        r = min(n, ref.PROBE_ROUNDS)
        assert np.array_equal(out[e, :, :r], S[:, :r]), e


@pytest.mark.skipif(not ref.available(), reason="reference harness not built")
@pytest.mark.parametrize("name,nenv,nedge,seed", [("plain", 12, 150, 31), ("uneven", 30, 200, 32),
                                                  ("multi_fetch", 12, 100, 33), ("multi_baxter", 10, 80, 34)])
def test_checker_matches_reference_cuda_path(checker, name, nenv, nedge, seed):
    robot = workload.robot_of(name)
    envs = workload.gen_envs(name, nenv, seed=seed)
    edges = workload.gen_edges(name, nedge, seed=seed)
    want = ref.check(envs, edges, robot=robot)
    checker.upload(envs)
    got = checker.check(edges, robot=robot)
    assert_parity(envs, edges, got, want, "vs reference CUDA", robot)
    # and the oracle against the reference (pins the oracle itself)
    assert_parity(envs, edges, orc.check(envs, edges, robot=robot), want, "oracle vs reference CUDA", robot)


@pytest.mark.skipif(not ref.available(), reason="reference harness not built")
def test_full_size_parity_vs_reference_cuda(checker):
    """Every (env, edge) pair of the full-size uneven workload (1000 envs x
    10000 edges, seed 0): both check orders against the reference's own public
    API batch_cc::batch_cc<Panda> (its CUDA kernel), each mismatch adjudicated
    by the FP64 penetration; none may lie beyond 1e-5 m of contact."""
    from bcc import mlp
    envs = workload.gen_envs("uneven", seed=0)
    edges = workload.gen_edges("uneven", seed=0)
    want = ref.check(envs, edges)
    checker.upload(envs)
    checker.mlp_set_params(mlp.init_params(3))
    for order in ("plain", "learned"):
        got = checker.check(edges, order=order)
        n_mis = assert_parity(envs, edges, got, want, "full size vs reference CUDA, %s order" % order)
        assert n_mis < 1e-4 * want.size, (order, n_mis)


def test_full_size_properties(checker):
    """Uneven workload at full size (1000 envs x 10000 edges): deterministic,
    and a random sample of pairs agrees with the oracle."""
    envs = workload.gen_envs("uneven", seed=0)
    edges = workload.gen_edges("uneven", seed=0)
    checker.upload(envs)
    a = checker.check(edges)
    b = checker.check(edges)
    assert np.array_equal(a, b)
    rng = np.random.default_rng(5)
    ei = rng.choice(len(edges), 60, replace=False)
    vi = rng.choice(envs.num_envs, 40, replace=False)
    sub_envs = envs.subset(vi)
    want = orc.check(sub_envs, edges[ei])
    assert_parity(sub_envs, edges[ei], a[np.ix_(ei, vi)], want, "full-size sample")
