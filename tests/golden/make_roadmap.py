"""Make the synthetic roadmap fixture of the CLI graph-mode tests.

The reference driver's graph.dot is not part of the reference tree (listed as a
missing large file), so a seeded stand-in is generated: a PRM-style graph of 40
Panda configurations uniform in the joint limits, each joined to its 3 nearest
neighbours, written the way Boost's write_graphviz writes a graph with a
`states` vertex property (plus an edge weight, a comment and one edge chain so
the reader's handling of those is exercised).

Usage: python tests/golden/make_roadmap.py
"""
import os

import numpy as np

here = os.path.dirname(os.path.abspath(__file__))
S_M = np.array([5.9342, 3.6652, 5.9342, 3.2289, 5.9342, 3.9095999999999997, 5.9342])
S_A = np.array([-2.9671, -1.8326, -2.9671, -3.1416, -2.9671, -0.0873, -2.9671])


def main():
    rng = np.random.default_rng(20261203)
    V = 40
    q = rng.uniform(0, 1, (V, 7)) * S_M + S_A
    d = np.linalg.norm(q[:, None] - q[None], axis=2)
    edges = []
    for i in range(V):
        for j in np.argsort(d[i])[1:4]:
            a, b = min(i, int(j)), max(i, int(j))
            if (a, b) not in edges:
                edges.append((a, b))
    lines = ["graph G {", "// synthetic roadmap: 40 Panda configurations, 3 nearest neighbours"]
    for i in range(V):
        lines.append('%d[states="%s"];' % (i, " ".join("%.9g" % v for v in q[i])))
    for k, (a, b) in enumerate(edges):
        lines.append("%d--%d [weight=%.6f];" % (a, b, d[a, b]) if k % 2 else "%d -- %d ;" % (a, b))
    # one chain statement adds two more edges
    lines.append("0 -- 39 -- 20;")
    lines.append("}")
    open(os.path.join(here, "roadmap_small.dot"), "w").write("\n".join(lines) + "\n")
    print("wrote", V, "vertices,", len(edges) + 2, "edges")


if __name__ == "__main__":
    main()
