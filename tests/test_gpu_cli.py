"""GPU test of the drop-in CLI driver (batch_cc <robot> <num_envs> <num_edges>
[file], and batch_cc <robot> <graph.dot> <scene.txt>) through the C++ facade:
its printed verdicts equal the oracle's and the reference CUDA path's on the
exact inputs it checked (dumped by the driver), for problem-file and scene-file
environments and roadmap-graph edges."""
import os
import subprocess

import numpy as np
import pytest

from bcc import EnvSet
from oracle import oracle as orc
from oracle import ref

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "batch-cc_b200", "batch_cc")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def read_dump(path):
    raw = open(path, "rb").read()
    N, E, dof = np.frombuffer(raw[:12], np.int32)
    counts = np.frombuffer(raw[12:12 + 12 * N], np.int32).reshape(N, 3)
    off = 12 + 12 * N
    envs = []
    for ns, nc, nb in counts:
        e = {}
        for key, k, w in (("spheres", ns, 4), ("capsules", nc, 8), ("cuboids", nb, 15)):
            e[key] = np.frombuffer(raw[off:off + 4 * k * w], np.float32).reshape(k, w)
            off += 4 * k * w
        envs.append(e)
    edges = np.frombuffer(raw[off:off + 4 * E * 2 * dof], np.float32).reshape(E, 2, dof)
    return EnvSet.from_lists(envs), edges.copy()


def run_cli(tmp_path, args):
    dump = str(tmp_path / "inputs.bin")
    env = dict(os.environ, BCC_DUMP_INPUTS=dump)
    r = subprocess.run([CLI] + args, capture_output=True, text=True, env=env, cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("Edge ")]
    got = np.array([[int(v) for v in l.split(":", 1)[1].split()] for l in lines], np.uint8)
    assert any(l.startswith("Throughput: ") and l.endswith(" edges/s") for l in r.stdout.splitlines())
    envs, edges = read_dump(dump)
    return got, envs, edges


@pytest.mark.parametrize("args", [["panda", "21", "64", "tests/golden/panda_problems_small.json"],
                                  ["panda", "8", "96", "tests/golden/scene_small.txt"],
                                  ["panda", "tests/golden/roadmap_small.dot", "tests/golden/scene_small.txt"]])
def test_cli_matches_oracle_and_reference(tmp_path, args):
    got, envs, edges = run_cli(tmp_path, args)
    assert got.shape == (len(edges), envs.num_envs)
    if not args[1].endswith(".dot"):
        assert got.shape[0] == int(args[2])
    n_mis, n_adj, bad = orc.adjudicate(envs, edges, got, orc.check(envs, edges))
    assert len(bad) == 0
    if ref.available():
        want = ref.check(envs, edges)
        n_mis, n_adj, bad = orc.adjudicate(envs, edges, got, want)
        assert len(bad) == 0
