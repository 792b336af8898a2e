"""GPU tests of the launch machinery: every launch configuration (tile size,
warps, persistent work queue), CUDA-graph replay and the autotuner give the
same verdicts, in both check orders."""
import numpy as np
import pytest

from bcc import mlp, workload

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(checker):
    envs = workload.gen_envs("uneven", 40, seed=51)
    edges = workload.gen_edges("uneven", 700, seed=51)
    checker.upload(envs)
    checker.mlp_set_params(mlp.init_params(3))
    checker.set_launch_config(edges_per_cta=128, warps=8, persistent=0, queue_min_items=128)
    base = checker.check(edges)
    return envs, edges, base


@pytest.mark.parametrize("lanes", [32, 16])
@pytest.mark.parametrize("tile", [1, 32, 77, 256])
@pytest.mark.parametrize("warps", [4, 8])
@pytest.mark.parametrize("persistent", [0, 1])
def test_launch_configs_agree(checker, case, tile, warps, persistent, lanes):
    """Every launch shape, with a whole warp or a half-warp (16 lanes) per
    walking pair, in both orders (the learned one inline and queued)."""
    envs, edges, base = case
    checker.upload(envs)
    checker.set_launch_config(edges_per_cta=tile, warps=warps, persistent=persistent, queue_min_items=64,
                              lanes=lanes, learned_mode=0, clusters=1)
    for order in ("plain", "learned"):
        assert np.array_equal(checker.check(edges, order=order), base), (tile, warps, persistent, lanes, order)
    checker.set_launch_config(learned_mode=1)
    assert np.array_equal(checker.check(edges, order="learned"), base), (tile, warps, persistent, lanes, "queued")
    checker.set_launch_config(learned_mode=0, lanes=32)


@pytest.mark.parametrize("name,robot", [("uneven", "panda"), ("multi_fetch", "fetch"), ("multi_baxter", "baxter")])
def test_half_warp_walk_keeps_verdicts_and_pairs(checker, name, robot):
    """16 lanes per walking pair: identical verdicts, and the work counters
    count every walked pair and every colliding pair once (robots with
    overhanging leaves keep the whole-warp walk)."""
    envs = workload.gen_envs(name, 30, seed=52)
    edges = workload.gen_edges(name, 400, seed=52)
    checker.upload(envs)
    cfg = checker.launch_config()
    work = {}
    try:
        checker.set_profiling(True, counters=True)
        for lanes in (32, 16):
            checker.set_launch_config(edges_per_cta=64, warps=4, persistent=0, lanes=lanes)
            v = checker.check(edges, robot=robot)
            work[lanes] = (v, checker.work_counters())
    finally:
        checker.set_profiling(False)
        checker.set_launch_config(**cfg)
    assert np.array_equal(work[32][0], work[16][0])
    for k in ("pairs", "candidates", "colliding"):
        assert work[32][1][k] == work[16][1][k], k


def test_graph_replay_agrees(checker, case):
    import torch
    envs, edges, base = case
    checker.upload(envs)
    checker.set_launch_config(edges_per_cta=64, warps=8, persistent=1, queue_min_items=128)
    d_edges = torch.from_numpy(edges).cuda()
    d_res = torch.zeros(base.shape, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    for order in ("plain", "learned"):
        for _ in range(3):  # capture, then replays
            d_res.zero_()
            checker.check_device(d_edges.data_ptr(), len(edges), d_res.data_ptr(), order=order, stream=s, graph=True)
            torch.cuda.synchronize()
            assert np.array_equal(d_res.cpu().numpy(), base), order
    # new edge contents: replayed, or re-captured when the sample total changed
    other = workload.gen_edges("uneven", 700, seed=52)
    d_edges.copy_(torch.from_numpy(other))
    checker.check_device(d_edges.data_ptr(), len(edges), d_res.data_ptr(), stream=s, graph=True)
    torch.cuda.synchronize()
    checker.set_launch_config(persistent=0)
    assert np.array_equal(d_res.cpu().numpy(), checker.check(other))


def test_autotune_picks_a_valid_config(checker, case):
    envs, edges, base = case
    checker.upload(envs)
    cfg = checker.autotune(edges, order="plain")
    assert cfg["edges_per_cta"] in (32, 64, 128, 256) and cfg["warps"] in (4, 8)
    assert np.array_equal(checker.check(edges), base)
    cfg = checker.autotune(edges, order="learned")
    # the learned order's shape, mode, clusters and queue threshold are swept
    assert cfg["edges_per_cta"] in (32, 64, 128, 256) and cfg["warps"] in (4, 8)
    assert cfg["learned_mode"] in (0, 1) and cfg["clusters"] in (1, 4, 8, 16) and cfg["lanes"] in (32, 16)
    if cfg["learned_mode"] == 1:
        assert cfg["queue_min_items"] in (64, 128, 256, 512, 1024, 2048, 4096)
    assert np.array_equal(checker.check(edges, order="learned"), base)
