"""GPU tests of the learned check order: the trained proposal never changes a
verdict, it is trained by the project's tensor-core kernels on checker labels,
its misprediction rate is measured, and it reduces the work spent on the pairs
a plain probe of their first sample leaves undecided."""
import numpy as np
import pytest

from bcc import mlp, workload
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


# Ranking is judged on the pairs queued with at least this many items left:
# long walks, where the order has room to matter.
RANK_MIN_ITEMS = 1024


@pytest.fixture(scope="module")
def trained(checker):
    """The network trained on the learned order's population (segments of the
    pairs the probe queues) of uneven environments and edges, seed 101; the
    ranking metrics are taken on seed-disjoint data (seed 102)."""
    train_envs = workload.gen_envs("uneven", 300, seed=101)
    train_edges = workload.gen_edges("uneven", 4000, seed=101)
    checker.mlp_set_params(mlp.init_params(7))
    checker.upload(train_envs)
    losses, pos, rows = checker.mlp_train_queued(train_edges, num_samples=1 << 20, queue_min_items=128, epochs=3,
                                                 batch=4096, lr=2e-3, seed=11)
    params = checker.mlp_get_params()
    checker.upload(workload.gen_envs("uneven", 400, seed=102))
    test_edges = workload.gen_edges("uneven", 4000, seed=102)
    ranking = checker.mlp_rank_metrics(test_edges, queue_min_items=RANK_MIN_ITEMS)
    checker.mlp_set_params(mlp.init_params(7))
    untrained = checker.mlp_rank_metrics(test_edges, queue_min_items=RANK_MIN_ITEMS)
    checker.mlp_set_params(params)
    return dict(losses=losses, pos=pos, rows=rows, params=params, ranking=ranking, untrained=untrained)


def test_training_learns(trained):
    """The training loss falls, and the population is the one the order acts on
    (a mix of colliding and free segments, not the ~87 % colliding samples of
    uniform draws)."""
    losses = trained["losses"]
    assert trained["rows"] > 10000
    assert losses[-1] < losses[0]
    assert 0.1 < trained["pos"] < 0.7, trained["pos"]


def test_learned_order_walks_less_than_plain(trained):
    """On held-out queued pairs, judged by exact per-sample checks: the
    learned walk reaches the first colliding sample in fewer sample ranks than
    the plain (reference) order, and no order beats the perfect one."""
    for m in (trained["ranking"], trained["untrained"]):
        assert m["queued_pairs"] > 100 and m["scored_segments"] >= 4 * m["queued_pairs"]
        assert 0.0 <= m["auc"] <= 1.0
        assert m["ranks_to_hit_perfect"] == 1.0
        assert m["ranks_to_hit_perfect"] <= m["ranks_to_hit_learned"]
        assert m["ranks_walked_perfect"] <= m["ranks_walked_plain"]
    m = trained["ranking"]
    assert m["ranks_to_hit_learned"] < m["ranks_to_hit_plain"], m
    assert m["ranks_walked_learned"] < m["ranks_walked_plain"], m


@pytest.fixture
def learned_mode(checker):
    """Sets the learned order's mode (0 inline, 1 queued) for one test and
    restores the launch configuration afterwards."""
    cfg = checker.launch_config()

    def use(mode, **kw):
        checker.set_launch_config(learned_mode=mode, **kw)
    yield use
    checker.set_launch_config(**cfg)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("name,nenv,nedge,seed", [("stress", 30, 400, 21), ("uneven", 30, 300, 22)])
def test_learned_order_keeps_verdicts(checker, trained, learned_mode, mode, name, nenv, nedge, seed):
    checker.mlp_set_params(trained["params"])
    learned_mode(mode, queue_min_items=128)
    envs = workload.gen_envs(name, nenv, seed=seed)
    edges = workload.gen_edges(name, nedge, seed=seed)
    checker.upload(envs)
    plain = checker.check(edges, order="plain")
    learned = checker.check(edges, order="learned")
    assert checker.last_learned_rows() > 0
    if mode == 1:  # every queued pair holds at least its 4 n >= 4 segment rows
        assert 0 < checker.last_learned_pairs() <= checker.last_learned_rows() // 4
    else:  # the inline order scores (cluster, segment) rows and queues nothing
        assert checker.last_learned_pairs() == 0
    # Same tests in a different order: identical verdicts.
    assert np.array_equal(plain, learned)
    n_mis, n_adj, bad = orc.adjudicate(envs, edges, learned, orc.check(envs, edges))
    assert len(bad) == 0


@pytest.mark.parametrize("clusters", [1, 3, 8, 64])
@pytest.mark.parametrize("graph", [False, True])
def test_inline_order_cluster_counts_keep_verdicts(checker, trained, learned_mode, clusters, graph):
    """The inline order with 1, 3, 8 and 64 environment clusters (64 > the 40
    environments: one cluster each), eager and replayed from a captured graph:
    verdicts stay the plain order's and the scored rows are clusters x
    segments."""
    checker.mlp_set_params(trained["params"])
    learned_mode(0, clusters=clusters)
    envs = workload.gen_envs("uneven", 40, seed=23)
    edges = workload.gen_edges("uneven", 500, seed=23)
    checker.upload(envs)
    plain = checker.check(edges, order="plain")
    segs = sum(4 * orc.edge_n(e[0], e[1]) for e in edges)
    for _ in range(2):
        assert np.array_equal(checker.check(edges, order="learned", graph=graph), plain)
        assert checker.last_learned_rows() == min(clusters, 40) * segs


def test_trained_network_saves_work(checker, trained):
    """What the learning adds: on held-out queued pairs the trained network's
    order reaches the first colliding sample in fewer sample ranks than the
    same pipeline with an untrained network (the method without the
    learning), and ranks the segments better (AUC)."""
    t, u = trained["ranking"], trained["untrained"]
    assert t["queued_pairs"] == u["queued_pairs"] and t["colliding_pairs"] == u["colliding_pairs"]
    assert t["ranks_to_hit_learned"] < u["ranks_to_hit_learned"], (t, u)
    assert t["auc"] > u["auc"], (t, u)


def test_work_counters_of_both_networks(checker, trained):
    """The same held-out check with the trained and an untrained network: the
    verdicts and the colliding count are the order's business of neither."""
    envs = workload.gen_envs("uneven", 200, seed=31)
    edges = workload.gen_edges("uneven", 3000, seed=31)
    checker.upload(envs)
    cfg = checker.launch_config()
    checker.set_launch_config(queue_min_items=RANK_MIN_ITEMS, learned_mode=1)
    checker.set_profiling(True, counters=True)
    work, verdicts = {}, {}
    try:
        for label, params in (("untrained", mlp.init_params(99)), ("trained", trained["params"])):
            checker.mlp_set_params(params)
            verdicts[label] = checker.check(edges, order="learned")
            work[label] = checker.work_counters()
    finally:
        checker.set_profiling(False)
        checker.set_launch_config(**cfg)
    assert np.array_equal(verdicts["trained"], verdicts["untrained"])
    assert work["trained"]["colliding"] == work["untrained"]["colliding"]
    assert work["trained"]["pairs"] == work["untrained"]["pairs"]


def test_trained_inline_order_walks_fewer_chunks(checker, trained):
    """What the learning adds to the order the tuner picks (inline, one
    cluster), on held-out environments and edges: the walk with the trained
    network takes fewer 32-item chunks per pair than with an untrained network
    (the order's structure alone), which takes fewer than the plain order."""
    envs = workload.gen_envs("uneven", 200, seed=31)
    edges = workload.gen_edges("uneven", 3000, seed=31)
    checker.upload(envs)
    cfg = checker.launch_config()
    checker.set_launch_config(learned_mode=0, clusters=1)
    checker.set_profiling(True, counters=True)
    chunks, verdicts = {}, {}
    try:
        verdicts["plain"] = checker.check(edges, order="plain")
        chunks["plain"] = checker.work_counters()["chunks"]
        for label, params in (("untrained", mlp.init_params(99)), ("trained", trained["params"])):
            checker.mlp_set_params(params)
            verdicts[label] = checker.check(edges, order="learned")
            chunks[label] = checker.work_counters()["chunks"]
    finally:
        checker.set_profiling(False)
        checker.set_launch_config(**cfg)
        checker.mlp_set_params(trained["params"])
    assert np.array_equal(verdicts["trained"], verdicts["plain"])
    assert np.array_equal(verdicts["untrained"], verdicts["plain"])
    assert chunks["trained"] < chunks["untrained"] < chunks["plain"], chunks


@pytest.mark.parametrize("row_cap", [3, 4, 64, 2000])
@pytest.mark.parametrize("graph", [False, True])
def test_row_budget_keeps_verdicts(checker, trained, learned_mode, row_cap, graph):
    """Queued order, a row budget smaller than the queue needs: pairs that find
    it spent (or whose segments would not fit) are walked on in plain order by
    the probe, the rest are scored and finished; verdicts stay the plain
    order's.  A budget below 4 rows queues nothing."""
    checker.mlp_set_params(trained["params"])
    learned_mode(1, queue_min_items=128)
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


@pytest.mark.parametrize("split", [1, 0])
@pytest.mark.parametrize("warps,persistent", [(1, 0), (2, 1), (4, 0), (8, 1)])
def test_finish_split_keeps_verdicts(checker, trained, warps, persistent, split):
    """Threshold 0 queues every pair still undecided after its first sample;
    the finish kernel splits each across 1, 2, 4 or 8 warps of its CTA
    (split = 1) or gives each its own warp (split = 0).  Verdicts stay the
    plain order's and the work counters still count every walked pair once."""
    checker.mlp_set_params(trained["params"])
    envs = workload.gen_envs("stress", 20, seed=51)
    edges = workload.gen_edges("stress", 300, seed=51)
    checker.upload(envs)
    cfg = checker.launch_config()
    try:
        checker.set_launch_config(edges_per_cta=64, warps=warps, persistent=persistent, queue_min_items=0,
                                  finish_split=split, learned_mode=1)
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


@pytest.mark.parametrize("mode,split", [(1, 1), (1, 0), (0, 0)])
@pytest.mark.parametrize("name", ["multi_fetch", "multi_baxter"])
def test_learned_order_overhang_robots(checker, name, mode, split):
    """Fetch and Baxter take the overhang-aware walk in the probe (queue
    decision inside the loop), in the split and one-warp finishes and in the
    inline order; with threshold 0 many pairs are queued, and every verdict
    must stay the plain order's."""
    robot = workload.robot_of(name)
    checker.mlp_set_params(mlp.init_params(61))
    envs = workload.gen_envs(name, 64, seed=61)
    edges = workload.gen_edges(name, 1000, seed=61)  # ~2 % of the pairs are collision-free
    checker.upload(envs)
    cfg = checker.launch_config()
    try:
        checker.set_launch_config(edges_per_cta=32, warps=4, persistent=0, queue_min_items=0, finish_split=split,
                                  learned_mode=mode)
        plain = checker.check(edges, order="plain", robot=robot)
        learned = checker.check(edges, order="learned", robot=robot)
        assert (checker.last_learned_pairs() > 0) if mode == 1 else (checker.last_learned_rows() > 0)
        assert np.array_equal(plain, learned)
    finally:
        checker.set_launch_config(**cfg)
