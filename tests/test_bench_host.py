"""CPU tests of bench.py's host-side pieces: both arms print the same config
dict, and the roofline's committed ncu counts parse from profiles/."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "batch-cc_b200"))
    import bench
    return bench


def test_both_arms_share_one_config():
    bench = _bench()
    a = bench.bench_config("uneven", 1000, 10000, 1)
    b = bench.bench_config("uneven", 1000, 10000, 1)
    assert a == b and a["envs"] == 1000 and a["edges_per_gpu"] == 10000 and "l2" in a
    assert "order" not in a  # the order is a top-level field of our arm's line, not part of the workload


def test_committed_counts_parse():
    bench = _bench()
    c = bench.committed_counts("uneven")
    assert c is not None
    for k in ("inst_per_pair", "ffma_per_pair", "fadd_per_pair", "fmul_per_pair", "dram_bytes_per_pair"):
        assert c[k] > 0, k
    assert 100 < c["inst_per_pair"] < 5000
    assert bench.committed_counts("no_such_workload") is None


def test_tuning_subset_outgrows_l2_like_the_full_workload():
    """The autotuner times configurations on all edges of the benchmark and the
    Fetch and Baxter workloads, and on enough edges of the stress workload that its
    sample table (about 43 KB of rows per Panda edge) exceeds the 126 MB L2."""
    bench = _bench()
    assert bench.tune_edges(10000, 1000) == 10000      # uneven Panda benchmark
    assert bench.tune_edges(5000, 500) == 5000         # Fetch / Baxter, 500 x 5000
    n = bench.tune_edges(100000, 10000)                # stress, 10 000 x 100 000
    assert 5000 <= n <= 10000
    assert n * 32 * 1.1 * 77 * 16 > 126e6
    assert bench.tune_edges(300, 10) == 300            # small cases: every edge
