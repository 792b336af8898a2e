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


@pytest.mark.parametrize("tile", [1, 32, 77, 256])
@pytest.mark.parametrize("warps", [4, 8])
@pytest.mark.parametrize("persistent", [0, 1])
def test_launch_configs_agree(checker, case, tile, warps, persistent):
    envs, edges, base = case
    checker.upload(envs)
    checker.set_launch_config(edges_per_cta=tile, warps=warps, persistent=persistent, queue_min_items=64)
    for order in ("plain", "learned"):
        assert np.array_equal(checker.check(edges, order=order), base), (tile, warps, persistent, order)


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
    assert cfg["learned_mode"] in (0, 1) and cfg["clusters"] in (1, 4, 8, 16)
    if cfg["learned_mode"] == 1:
        assert cfg["queue_min_items"] in (64, 128, 256, 512, 1024, 2048, 4096)
    assert np.array_equal(checker.check(edges, order="learned"), base)
