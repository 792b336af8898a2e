"""CPU tests of the C++ drop-in (headers under include/src, the CLI driver and
its loaders): Halton edges, joint-limit scaling, problem-file and scene
loading, CLI argument handling."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
CLI = os.path.join(ROOT, "batch-cc_b200", "batch_cc")


@pytest.fixture(scope="module")
def dropin_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("dropin") / "dropin_test")
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I",
                           os.path.join(ROOT, "batch-cc_b200", "cli"), os.path.join(ROOT, "tests", "cpp", "dropin_test.cpp"),
                           "-o", out])
    return out


def halton_reference(n, bases):
    """The incremental Halton recurrence in float32, written independently."""
    f = np.float32
    num = [f(0)] * len(bases)
    den = [f(1)] * len(bases)
    rows = []
    for _ in range(n):
        row = []
        for i, b in enumerate(bases):
            b = f(b)
            x = f(den[i] - num[i])
            if x == f(1):
                den[i] = f(np.floor(f(den[i] * b)))
                num[i] = f(1)
            else:
                y = f(np.floor(f(den[i] / b)))
                while x <= y:
                    y = f(np.floor(f(y / b)))
                num[i] = f(f(np.floor(f(f(b + f(1)) * y))) - x)
            row.append(f(num[i] / den[i]))
        rows.append(row)
    return np.array(rows, np.float32)


def test_halton_matches_recurrence(dropin_bin):
    out = subprocess.check_output([dropin_bin, "halton"], text=True)
    got = np.array([[float(v) for v in l.split()] for l in out.strip().splitlines()], np.float32)
    want = halton_reference(2000, [3, 5, 7, 11, 13, 17, 19])
    assert np.array_equal(got, want)
    assert np.allclose(got[:4, 0], [1 / 3, 2 / 3, 1 / 9, 4 / 9])


def test_halton_matches_reference_header(tmp_path):
    """The drop-in header against the reference's own src/random/halton.hh:
    1,000,010 draws per dimension (7, 8, 14), past the restart after
    max_iterations, identical bit for bit (fixture made by
    tests/golden/make_halton.py from the reference header)."""
    exe = str(tmp_path / "halton_draws")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "halton_draws.cpp"), "-o", exe])
    got = subprocess.check_output([exe], text=True)
    want = open(os.path.join(GOLDEN, "halton_reference.txt")).read()
    assert got == want


def test_scale_cfg(dropin_bin):
    out = subprocess.check_output([dropin_bin, "scale"], text=True)
    got = np.array([float(v) for v in out.split()], np.float32)
    from bcc.workload import LIMITS
    s_m, s_a = LIMITS["panda"]
    u = np.array([0, 0.25, 0.5, 0.75, 1, 0.1, 0.9], np.float32)
    assert np.allclose(got, u * s_m + s_a, atol=1e-6)


def test_mbm_loader_counts(dropin_bin):
    path = os.path.join(GOLDEN, "panda_problems_small.json")
    out = subprocess.check_output([dropin_bin, "mbm", path], text=True).strip().splitlines()
    d = json.load(open(path))
    want = []
    for fam in sorted(d["problems"]):
        for p in d["problems"][fam]:
            if not p["valid"]:
                continue
            ncyl = len(p["cylinder"])
            want.append((len(p["sphere"]), 0 if fam == "box" else ncyl, len(p["box"]) + (ncyl if fam == "box" else 0)))
    got = [tuple(int(v) for v in l.split()) for l in out[:-1]]
    assert got == want
    assert out[-1] == "moved 1 1"


def test_scene_loader_counts(dropin_bin):
    out = subprocess.check_output([dropin_bin, "scene", os.path.join(GOLDEN, "scene_small.txt"), "8"],
                                  text=True).strip().splitlines()
    # 2 shared OBJECT boxes + 3 obstacle boxes + 1 target cylinder per environment
    assert [tuple(int(v) for v in l.split()) for l in out[:-1]] == [(0, 1, 5)] * 8


def test_cli_usage_and_unknown_robot():
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert r.returncode == 1 and r.stdout.startswith("Usage:")
    r = subprocess.run([CLI, "xarm7", "1", "1", os.devnull], capture_output=True, text=True)
    assert r.returncode == 255 and "Unknown robot name" in r.stdout


def _roadmap():
    """Vertices and edges of tests/golden/roadmap_small.dot, read with regexes."""
    import re
    text = open(os.path.join(ROOT, "tests", "golden", "roadmap_small.dot")).read()
    states = {int(m.group(1)): [float(v) for v in m.group(2).split()]
              for m in re.finditer(r'^(\d+)\[states="([^"]*)"\];$', text, re.M)}
    edges = []
    for line in text.splitlines():
        if "--" in line:
            ids = [int(t) for t in re.findall(r"\d+(?=\s*(?:--|;|\[))", line.split("[")[0] + ";")]
            edges += list(zip(ids[:-1], ids[1:]))
    return states, edges


def test_cli_graph_mode_reads_the_roadmap(tmp_path):
    """`batch_cc <robot> <graph.dot> <scene.txt>`: edges in file order with their
    vertices' states (chains included), 200 scene environments -- checked on the
    inputs the driver dumps before it checks (without a GPU the check then fails)."""
    import numpy as np
    dump = str(tmp_path / "inputs.bin")
    env = dict(os.environ, BCC_DUMP_INPUTS=dump)
    r = subprocess.run([CLI, "panda", "tests/golden/roadmap_small.dot", "tests/golden/scene_small.txt"],
                       capture_output=True, text=True, env=env, cwd=ROOT, timeout=120)
    states, edges = _roadmap()
    assert "Number of edges: %d" % len(edges) in r.stdout
    assert "Number of environments: 200" in r.stdout
    raw = open(dump, "rb").read()
    N, E, dof = np.frombuffer(raw[:12], np.int32)
    assert (N, E, dof) == (200, len(edges), 7)
    got = np.frombuffer(raw[-4 * E * 2 * dof:], np.float32).reshape(E, 2, dof)
    want = np.array([[states[a], states[b]] for a, b in edges], np.float32)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("text,msg", [("digraph G { a -> b }", "fewer states"),
                                      ("graph G { subgraph s { a } }", "subgraphs"),
                                      ("graph G { a [states=\"1 2\"", "unterminated"),
                                      ("tree G { }", "expected graph")])
def test_cli_graph_mode_rejects_bad_files(tmp_path, text, msg):
    p = tmp_path / "g.dot"
    p.write_text(text)
    r = subprocess.run([CLI, "panda", str(p), "tests/golden/scene_small.txt"], capture_output=True, text=True,
                       cwd=ROOT, timeout=60)
    assert r.returncode == 2 and msg in r.stderr, (r.returncode, r.stderr)
