"""Multi-process paths of bench.py on CPU (gloo, world size 2): the reference
arm under torchrun, the max-over-ranks reduction and per-rank edge sets.  The
GPU arm shards the same way over NCCL; nothing here needs a GPU."""
import json
import os
import socket
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_under_torchrun_two_ranks():
    """Rank 0 alone runs the reference arm and prints one JSON line; rank 1
    exits 0 without output."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--envs", "4", "--edges", "60"]
    r = subprocess.run(["timeout", "-k", "30", "240"] + cmd, capture_output=True, text=True, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "edges/s"
    assert d["cpu_baseline"]["cores"] >= 1 and d["e2e"]["h2d_bytes_per_step"] == 0


def _worker(rank, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "batch-cc_b200"))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    got = bench.max_over_ranks(dist, 1.5 + rank, "cpu")
    e = bench.rank_edges("uneven", 20, rank)
    np.save(os.path.join(out, "edges%d.npy" % rank), e)
    with open(os.path.join(out, "max%d.txt" % rank), "w") as f:
        f.write(repr(got))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_rank_edge_sets(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert [float(open(tmp_path / ("max%d.txt" % r)).read()) for r in (0, 1)] == [2.5, 2.5]
    e0, e1 = np.load(tmp_path / "edges0.npy"), np.load(tmp_path / "edges1.npy")
    assert e0.shape == e1.shape == (20, 2, 7) and not np.array_equal(e0, e1)
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.25, "cpu") == 3.25
