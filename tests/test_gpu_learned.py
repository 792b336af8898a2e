"""GPU tests of the learned check order: the trained proposal never changes a
verdict, it is trained by the project's tensor-core kernels on checker labels,
its misprediction rate is measured, and it reduces the work spent on the pairs
a plain probe of their first sample leaves undecided."""
import numpy as np
import pytest

from bcc import mlp, workload
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained(checker):
    train_envs = workload.gen_envs("stress", 64, seed=101)
    train_edges = workload.gen_edges("stress", 3000, seed=101)
    checker.mlp_set_params(mlp.init_params(7))
    checker.upload(train_envs)
    losses, pos = checker.mlp_train(train_edges, num_samples=1 << 19, epochs=3, batch=8192, lr=2e-3, seed=11)
    metrics = checker.mlp_evaluate(workload.gen_edges("stress", 1000, seed=102), 1 << 16, seed=12)
    return dict(losses=losses, pos=pos, metrics=metrics, params=checker.mlp_get_params())


def test_training_learns(trained):
    losses, m = trained["losses"], trained["metrics"]
    assert losses[-1] < losses[0]
    base = min(m["positive"], 1 - m["positive"])  # error of the constant predictor
    assert m["mispredict"] < base, (m, base)


@pytest.mark.parametrize("name,nenv,nedge,seed", [("stress", 30, 400, 21), ("uneven", 30, 300, 22)])
def test_learned_order_keeps_verdicts(checker, trained, name, nenv, nedge, seed):
    checker.mlp_set_params(trained["params"])
    envs = workload.gen_envs(name, nenv, seed=seed)
    edges = workload.gen_edges(name, nedge, seed=seed)
    checker.upload(envs)
    plain = checker.check(edges, order="plain")
    learned = checker.check(edges, order="learned")
    assert checker.last_learned_rows() > 0
    # every queued pair holds at least its 4 n >= 4 segment rows
    assert 0 < checker.last_learned_pairs() <= checker.last_learned_rows() // 4
    # Same tests in a different order: identical verdicts.
    assert np.array_equal(plain, learned)
    n_mis, n_adj, bad = orc.adjudicate(envs, edges, learned, orc.check(envs, edges))
    assert len(bad) == 0


def test_trained_network_saves_work(checker, trained):
    """Chunks walked on the stress workload: trained proposal vs the same
    pipeline with an untrained network (the method without the learning)."""
    envs = workload.gen_envs("stress", 40, seed=31)
    edges = workload.gen_edges("stress", 1500, seed=31)
    checker.upload(envs)
    checker.set_profiling(True, counters=True)
    work = {}
    for label, params in (("untrained", mlp.init_params(99)), ("trained", trained["params"])):
        checker.mlp_set_params(params)
        checker.check(edges, order="learned")
        work[label] = checker.work_counters()
    checker.set_profiling(False)
    assert work["trained"]["colliding"] == work["untrained"]["colliding"]
    assert work["trained"]["chunks"] <= work["untrained"]["chunks"], work


@pytest.mark.parametrize("row_cap", [3, 4, 64, 2000])
@pytest.mark.parametrize("graph", [False, True])
def test_row_budget_keeps_verdicts(checker, trained, row_cap, graph):
    """A row budget smaller than the queue needs: pairs that find it spent (or
    whose segments would not fit) are walked on in plain order by the probe,
    the rest are scored and finished; verdicts stay the plain order's.  A budget
    below 4 rows queues nothing."""
    checker.mlp_set_params(trained["params"])
    envs = workload.gen_envs("stress", 24, seed=41)
    edges = workload.gen_edges("stress", 400, seed=41)
    checker.upload(envs)
    plain = checker.check(edges, order="plain")
    for _ in range(2):  # the second call replays the captured graph when graph=True
        learned = checker.check(edges, order="learned", graph=graph, row_cap=row_cap)
        assert np.array_equal(plain, learned)
        rows = checker.last_learned_rows()
        assert 0 <= rows <= row_cap
        if row_cap < 4:
            assert rows == 0
    # the default budget scores more rows than any of the small ones
    checker.check(edges, order="learned")
    assert checker.last_learned_rows() > min(row_cap, 64)


def test_negative_row_budget_is_rejected(checker, trained):
    checker.mlp_set_params(trained["params"])
    checker.upload(workload.gen_envs("stress", 4, seed=42))
    with pytest.raises(Exception, match="learned_row_cap"):
        checker.check(workload.gen_edges("stress", 10, seed=42), order="learned", row_cap=-1)


@pytest.mark.parametrize("warps,persistent", [(1, 0), (2, 1), (4, 0), (8, 1)])
def test_finish_split_keeps_verdicts(checker, trained, warps, persistent):
    """Threshold 0 queues every pair still undecided after its first sample;
    the finish kernel splits each across 1, 2, 4 or 8 warps of its CTA.
    Verdicts stay the plain order's and the work counters still count every
    walked pair once."""
    checker.mlp_set_params(trained["params"])
    envs = workload.gen_envs("stress", 20, seed=51)
    edges = workload.gen_edges("stress", 300, seed=51)
    checker.upload(envs)
    cfg = checker.launch_config()
    try:
        checker.set_launch_config(edges_per_cta=64, warps=warps, persistent=persistent, queue_min_items=0)
        checker.set_profiling(True, counters=True)
        plain = checker.check(edges, order="plain")
        work_plain = checker.work_counters()
        learned = checker.check(edges, order="learned")
        work_learned = checker.work_counters()
        checker.set_profiling(False)
        assert np.array_equal(plain, learned)
        assert checker.last_learned_pairs() > 0
        assert work_learned["pairs"] == work_plain["pairs"]
        assert work_learned["colliding"] == work_plain["colliding"]
    finally:
        checker.set_profiling(False)
        checker.set_launch_config(**cfg)


@pytest.mark.parametrize("name", ["multi_fetch", "multi_baxter"])
def test_learned_order_overhang_robots(checker, name):
    """Fetch and Baxter take the overhang-aware walk in the probe (queue
    decision inside the loop) and in the split finish; with threshold 0 many
    pairs are queued, and every verdict must stay the plain order's."""
    robot = workload.robot_of(name)
    checker.mlp_set_params(mlp.init_params(61))
    envs = workload.gen_envs(name, 64, seed=61)
    edges = workload.gen_edges(name, 1000, seed=61)  # ~2 % of the pairs are collision-free
    checker.upload(envs)
    cfg = checker.launch_config()
    try:
        checker.set_launch_config(edges_per_cta=32, warps=4, persistent=0, queue_min_items=0)
        plain = checker.check(edges, order="plain", robot=robot)
        learned = checker.check(edges, order="learned", robot=robot)
        assert checker.last_learned_pairs() > 0
        assert np.array_equal(plain, learned)
    finally:
        checker.set_launch_config(**cfg)
