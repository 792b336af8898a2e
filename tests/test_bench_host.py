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
